// The surrogate network: MLP 4 -> 256 -> 256 -> 256 -> 17 (SiLU), BF16 operands,
// FP32 accumulation, trained and evaluated by this file's kernels.
//
// Output 0 is the (normalised) LLE, outputs 1..16 the logits of the 16-way
// peak-count regime class.  Parameters live as FP32 masters (Adam state next to
// them) plus BF16 copies that feed the tensor cores.  Prediction over a whole
// grid runs as one fused tcgen05 kernel (mlp_tc.cuh).  Training and the
// prediction of explicit feature rows put every matrix product -- forward,
// input gradients, weight gradients -- through one tensor-core
// GEMM: mma.sync m16n8k16 BF16 x BF16 -> FP32, 64x64 CTA tiles, operands staged
// in shared memory in their memory order (k- or m/n-contiguous) by double-buffered
// 16-byte cp.async copies and read with ldmatrix (.trans for m/n-contiguous
// tiles), so transposed products need no copies, and fused epilogues (bias, SiLU
// with the pre-activation kept,
// SiLU-derivative product for the backward pass, FP32 and/or BF16 stores).  A
// training step (minibatch gather, 4 forward GEMMs, loss, 7 backward GEMMs, bias
// reductions, Adam) is captured once as a CUDA graph and replayed.
#include <cuda_bf16.h>
#include <math.h>
#include <string.h>

#include <vector>

#include "mlp.cuh"

namespace cbf {

constexpr int kIn = 4, kHid = 256, kOut = 17, kClasses = 16;

namespace {

typedef __nv_bfloat16 bf16;

// Parameter layout of the flat FP32 buffer: W1[256x4] b1 W2[256x256] b2 W3 b3 W4[17x256] b4.
constexpr long long kW1 = 0, kB1 = kW1 + kHid * kIn;
constexpr long long kW2 = kB1 + kHid, kB2 = kW2 + kHid * kHid;
constexpr long long kW3 = kB2 + kHid, kB3 = kW3 + kHid * kHid;
constexpr long long kW4 = kB3 + kHid, kB4 = kW4 + kOut * kHid;
constexpr long long kNumParams = kB4 + kOut;

struct GemmDesc {
    const bf16* A;       // element (m, k) at A[m*a_m + k*a_k]
    long long a_m, a_k;
    const bf16* B;       // element (k, n) at B[k*b_k + n*b_n]
    long long b_k, b_n;
    int M, N, K;
    const float* bias;   // [N] or null
    int act;             // 1: SiLU
    const float* dz;     // optional: result *= silu'(dz[m*ldz + n])
    long long ldz;
    float* Z;            // optional: pre-activation (after bias)
    long long ldZ;
    float* C;            // optional FP32 result at C[m*c_m + n*c_n]
    long long c_m, c_n;
    bf16* Cb;            // optional BF16 result, row-major with ldCb
    long long ldCb;
    int splitK;          // >1: FP32 partials over K slices into ws[z][M*N], then summed
    float* ws;
};

constexpr int BM = 64, BN = 64, BK = 32, kGemmThreads = 128;

__device__ __forceinline__ float silu(float z) { return z / (1.0f + __expf(-z)); }
__device__ __forceinline__ float silu_grad(float z)
{
    const float s = 1.0f / (1.0f + __expf(-z));
    return s * (1.0f + z * (1.0f - s));
}

__device__ __forceinline__ void mma_bf16(float (&c)[4], const uint32_t (&a)[4], const uint32_t (&b)[2])
{
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
        "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// Operand staging modes: K-major (k contiguous in memory), MN-major (m or n
// contiguous) -- both 16-byte cp.async copies, double-buffered -- or scalar
// loads for operands whose rows are not 16-byte multiples (K = 4, N = 17).
enum { kScalar = 0, kKMajor = 1, kMNMajor = 2 };
constexpr int kTileElems = BM * (BK + 8);  // >= BK * (BM + 8): both tile shapes fit
constexpr int kPitchK = BK + 8;            // K-major tile [64][40]: 80-byte rows
constexpr int kPitchMN = BM + 8;           // MN-major tile [32][72]: 144-byte rows

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, bool valid)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    const int bytes = valid ? 16 : 0;  // 0: zero-fill, nothing read
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;\n" ::); }

__device__ __forceinline__ void ldsm_x4(uint32_t (&r)[4], const bf16* p)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(p);
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(s));
}
__device__ __forceinline__ void ldsm_x4_t(uint32_t (&r)[4], const bf16* p)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(p);
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(s));
}

// One operand tile (rows r0 .. r0+64 of the M or N dimension, k0 .. k0+32) into
// shared memory.  Element (r, k) of the operand is at P[r*sr + k*sk].
template <int MODE>
__device__ __forceinline__ void load_tile(bf16* sm, const bf16* P, long long sr, long long sk, int R, int r0,
                                          int k0, int kEnd)
{
    if (MODE == kKMajor) {  // sm[r][k]
        for (int c = threadIdx.x; c < BM * (BK / 8); c += kGemmThreads) {
            const int r = c / (BK / 8), kc = (c % (BK / 8)) * 8;
            const bool v = r0 + r < R && k0 + kc < kEnd;
            cp_async16(sm + r * kPitchK + kc, v ? P + (long long)(r0 + r) * sr + (k0 + kc) : P, v);
        }
    } else if (MODE == kMNMajor) {  // sm[k][r]
        for (int c = threadIdx.x; c < BK * (BM / 8); c += kGemmThreads) {
            const int k = c / (BM / 8), rc = (c % (BM / 8)) * 8;
            const bool v = k0 + k < kEnd && r0 + rc < R;
            cp_async16(sm + k * kPitchMN + rc, v ? P + (long long)(k0 + k) * sk + (r0 + rc) : P, v);
        }
    } else {  // scalar, into the K-major shape; walks the unit-stride dimension fastest
        const bf16 zero = __float2bfloat16_rn(0.f);
        const bool kFast = sk == 1;
        for (int e = threadIdx.x; e < BM * BK; e += kGemmThreads) {
            const int r = kFast ? e / BK : e % BM, c = kFast ? e % BK : e / BM;
            const int rr = r0 + r, k = k0 + c;
            sm[r * kPitchK + c] = (rr < R && k < kEnd) ? P[rr * sr + k * sk] : zero;
        }
    }
}

template <int AM, int BMD>
__global__ void __launch_bounds__(kGemmThreads) gemm_bf16_kernel(const GemmDesc g)
{
    __shared__ __align__(128) bf16 smA[2][kTileElems];
    __shared__ __align__(128) bf16 smB[2][kTileElems];
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
    const int gq = lane >> 2, tq = lane & 3;
    const int lq = lane >> 3, l8 = lane & 7;  // ldmatrix: matrix and row of this lane's address
    float acc[2][4][4];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int v = 0; v < 4; ++v) acc[i][j][v] = 0.f;

    // K slice of this CTA (split-K: gridDim.z slices of whole BK blocks)
    const int kPer = ((g.K + BK - 1) / BK + gridDim.z - 1) / gridDim.z * BK;
    const int kBeg = blockIdx.z * kPer;
    const int kEnd = min(g.K, kBeg + kPer);
    const int nk = kEnd > kBeg ? (kEnd - kBeg + BK - 1) / BK : 0;

    if (nk > 0) {
        load_tile<AM>(smA[0], g.A, g.a_m, g.a_k, g.M, m0, kBeg, kEnd);
        load_tile<BMD>(smB[0], g.B, g.b_n, g.b_k, g.N, n0, kBeg, kEnd);
    }
    cp_async_commit();
    for (int it = 0; it < nk; ++it) {
        const int cur = it & 1;
        if (it + 1 < nk) {
            const int k1 = kBeg + (it + 1) * BK;
            load_tile<AM>(smA[cur ^ 1], g.A, g.a_m, g.a_k, g.M, m0, k1, kEnd);
            load_tile<BMD>(smB[cur ^ 1], g.B, g.b_n, g.b_k, g.N, n0, k1, kEnd);
        }
        cp_async_commit();
        cp_async_wait1();
        __syncthreads();
        const bf16* As = smA[cur];
        const bf16* Bs = smB[cur];
#pragma unroll
        for (int kk = 0; kk < BK; kk += 16) {
            uint32_t a[2][4], b[4][2];
#pragma unroll
            for (int mi = 0; mi < 2; ++mi) {
                const int mb = wm + mi * 16;
                if (AM == kMNMajor)
                    ldsm_x4_t(a[mi], As + (kk + (lq >> 1) * 8 + l8) * kPitchMN + mb + (lq & 1) * 8);
                else
                    ldsm_x4(a[mi], As + (mb + (lq & 1) * 8 + l8) * kPitchK + kk + (lq >> 1) * 8);
            }
#pragma unroll
            for (int np = 0; np < 2; ++np) {
                const int nb = wn + np * 16;
                uint32_t r[4];
                if (BMD == kMNMajor)
                    ldsm_x4_t(r, Bs + (kk + (lq & 1) * 8 + l8) * kPitchMN + nb + (lq >> 1) * 8);
                else
                    ldsm_x4(r, Bs + (nb + (lq >> 1) * 8 + l8) * kPitchK + kk + (lq & 1) * 8);
                b[2 * np][0] = r[0];
                b[2 * np][1] = r[1];
                b[2 * np + 1][0] = r[2];
                b[2 * np + 1][1] = r[3];
            }
#pragma unroll
            for (int mi = 0; mi < 2; ++mi)
#pragma unroll
                for (int ni = 0; ni < 4; ++ni) mma_bf16(acc[mi][ni], a[mi], b[ni]);
        }
        __syncthreads();
    }

#pragma unroll
    for (int mi = 0; mi < 2; ++mi)
#pragma unroll
        for (int ni = 0; ni < 4; ++ni)
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                const int m = m0 + wm + mi * 16 + gq + (v >= 2 ? 8 : 0);
                const int n = n0 + wn + ni * 8 + 2 * tq + (v & 1);
                if (m >= g.M || n >= g.N) continue;
                float z = acc[mi][ni][v];
                if (g.splitK > 1) {
                    g.ws[((long long)blockIdx.z * g.M + m) * g.N + n] = z;
                    continue;
                }
                if (g.bias) z += g.bias[n];
                if (g.Z) g.Z[m * g.ldZ + n] = z;
                if (g.dz) z *= silu_grad(g.dz[m * g.ldz + n]);
                const float y = g.act ? silu(z) : z;
                if (g.C) g.C[m * g.c_m + n * g.c_n] = y;
                if (g.Cb) g.Cb[m * g.ldCb + n] = __float2bfloat16_rn(y);
            }
}

bool aligned16(const void* p) { return ((uintptr_t)p & 15) == 0; }

// Staging mode of an operand: element (r, k) at P[r*sr + k*sk], R rows.
int stage_mode(const void* P, long long sr, long long sk, int R, int K)
{
    if (!aligned16(P)) return kScalar;
    if (sk == 1 && sr % 8 == 0 && K % 8 == 0) return kKMajor;
    if (sr == 1 && sk % 8 == 0 && R % 8 == 0) return kMNMajor;
    return kScalar;
}

template <int AM>
void launch_gemm_b(int bm, dim3 grid, const GemmDesc& g, cudaStream_t s)
{
    switch (bm) {
    case kKMajor: gemm_bf16_kernel<AM, kKMajor><<<grid, kGemmThreads, 0, s>>>(g); break;
    case kMNMajor: gemm_bf16_kernel<AM, kMNMajor><<<grid, kGemmThreads, 0, s>>>(g); break;
    default: gemm_bf16_kernel<AM, kScalar><<<grid, kGemmThreads, 0, s>>>(g); break;
    }
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

cudaError_t gemm(const GemmDesc& g, cudaStream_t s)
{
    const int splits = g.splitK > 1 ? g.splitK : 1;
    dim3 grid((g.N + BN - 1) / BN, (g.M + BM - 1) / BM, splits);
    if (grid.x == 0 || grid.y == 0) return cudaSuccess;
    const int am = stage_mode(g.A, g.a_m, g.a_k, g.M, g.K);
    const int bm = stage_mode(g.B, g.b_n, g.b_k, g.N, g.K);
    switch (am) {
    case kKMajor: launch_gemm_b<kKMajor>(bm, grid, g, s); break;
    case kMNMajor: launch_gemm_b<kMNMajor>(bm, grid, g, s); break;
    default: launch_gemm_b<kScalar>(bm, grid, g, s); break;
    }
    note_launch();
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess || splits == 1) return e;
    const long long MN = (long long)g.M * g.N;
    splitk_reduce_kernel<<<(unsigned)((MN + 255) / 256), 256, 0, s>>>(g.ws, splits, g.M, g.N, g.C, g.c_m, g.c_n);
    note_launch();
    return cudaGetLastError();
}

GemmDesc gdesc()
{
    GemmDesc g;
    memset(&g, 0, sizeof(g));
    return g;
}

// ---- element-wise kernels -------------------------------------------------

__device__ __forceinline__ unsigned long long mix64(unsigned long long z)
{
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// Minibatch of B rows drawn uniformly (with replacement) from N, keyed by the
// device step counter so a replayed graph draws a new batch every step.
__global__ void gather_kernel(const float* __restrict__ X, const float* __restrict__ ylle,
                              const int* __restrict__ ycls, long long N, int B,
                              const unsigned long long* step, unsigned long long seed,
                              bf16* __restrict__ xb, float* __restrict__ bl, int* __restrict__ bc)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= B) return;
    const unsigned long long h = mix64(seed ^ mix64(*step * 0x100000001B3ull + (unsigned long long)r));
    const long long i = (long long)(h % (unsigned long long)N);
#pragma unroll
    for (int f = 0; f < kIn; ++f) xb[(long long)r * kIn + f] = __float2bfloat16_rn(X[i * kIn + f]);
    bl[r] = ylle[i];
    bc[r] = ycls[i];
}

// Loss: mean squared error on output 0 (normalised LLE) + cross-entropy of
// outputs 1..16; writes dLoss/dOut (FP32 and BF16) and accumulates the loss.
__global__ void loss_kernel(const float* __restrict__ out, const float* __restrict__ yl,
                            const int* __restrict__ yc, int B, float wLle, float* __restrict__ dOut,
                            bf16* __restrict__ dOutB, float* __restrict__ lossAcc)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= B) return;
    const float* o = out + (long long)r * kOut;
    float* d = dOut + (long long)r * kOut;
    const float invB = 1.0f / (float)B;
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
    for (int c = 0; c < kOut; ++c) dOutB[(long long)r * kOut + c] = __float2bfloat16_rn(d[c]);
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

// Adam on the flat FP32 parameters; refreshes the BF16 weight copies.
__global__ void adam_kernel(float* __restrict__ p, const float* __restrict__ gr, float* __restrict__ m1,
                            float* __restrict__ m2, bf16* __restrict__ pb, long long n, float lr0,
                            int horizon, float b1, float b2, float eps, const unsigned long long* step)
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
        pb[i] = __float2bfloat16_rn(w);
    }
}

__global__ void bump_kernel(unsigned long long* step) { *step += 1; }

__global__ void to_bf16_kernel(const float* __restrict__ a, bf16* __restrict__ b, long long n)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = __float2bfloat16_rn(a[i]);
}

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

__device__ __forceinline__ void point_features(const FeatureSpec& f, long long g, float (&x)[kIn])
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
    float x[kIn];
    point_features(f, idx[k], x);
#pragma unroll
    for (int i = 0; i < kIn; ++i) X[k * kIn + i] = x[i];
}

#include "mlp_tc.cuh"

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

struct Mlp {
    int B = 0;               // training batch
    unsigned long long seed = 0;
    float* params = nullptr;  // FP32 masters (kNumParams)
    float* grads = nullptr;
    float* m1 = nullptr;
    float* m2 = nullptr;
    bf16* pb = nullptr;       // BF16 copies
    // batch buffers
    bf16* xb = nullptr;
    float* yl = nullptr;
    int* yc = nullptr;
    float *z1 = nullptr, *z2 = nullptr, *z3 = nullptr;
    bf16 *h1 = nullptr, *h2 = nullptr, *h3 = nullptr;
    float* out = nullptr;
    float* dOut = nullptr;
    bf16* dOutB = nullptr;
    float* dz = nullptr;      // FP32 dZ of the layer being reduced
    bf16 *dz3 = nullptr, *dz2 = nullptr, *dz1 = nullptr;
    float* loss = nullptr;
    float* ws = nullptr;      // split-K partials
    unsigned long long* step = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    const float* gX = nullptr;  // training set the graph was captured for
    long long gN = 0;
    float gLr = 0.f;
    int gHorizon = 0;
    float gW = 0.f;
    unsigned long long gSeed = 0;
    // inference workspace (rows per chunk = kPredRows), no pre-activations
    bf16 *pxb = nullptr, *ph1 = nullptr, *ph2 = nullptr, *ph3 = nullptr;
    float* pout = nullptr;
    // grid prediction on tcgen05: weights in the shared-memory operand layout
    unsigned char* wpack = nullptr;
    int* tcErr = nullptr;
};

constexpr int kPredRows = 262144;

namespace {
cudaError_t pred_workspace(Mlp* m)
{
    if (m->pxb) return cudaSuccess;
    cudaError_t e = cudaMalloc((void**)&m->pxb, (size_t)kPredRows * kIn * sizeof(bf16));
    if (e == cudaSuccess) e = cudaMalloc((void**)&m->ph1, (size_t)kPredRows * kHid * sizeof(bf16));
    if (e == cudaSuccess) e = cudaMalloc((void**)&m->ph2, (size_t)kPredRows * kHid * sizeof(bf16));
    if (e == cudaSuccess) e = cudaMalloc((void**)&m->ph3, (size_t)kPredRows * kHid * sizeof(bf16));
    if (e == cudaSuccess) e = cudaMalloc((void**)&m->pout, (size_t)kPredRows * kOut * sizeof(float));
    return e;
}
}  // namespace

namespace {

// Forward on a batch already in xb (n rows).  Keeps Z for the backward pass.
cudaError_t forward(Mlp& m, int n, const bf16* xb, float* out, float* z1, float* z2, float* z3,
                    bf16* h1, bf16* h2, bf16* h3, cudaStream_t s)
{
    const bf16* W = m.pb;
    cudaError_t e;
    GemmDesc g = gdesc();
    g.A = xb; g.a_m = kIn; g.a_k = 1;
    g.B = W + kW1; g.b_k = 1; g.b_n = kIn;
    g.M = n; g.N = kHid; g.K = kIn;
    g.bias = m.params + kB1; g.act = 1; g.Z = z1; g.ldZ = kHid; g.Cb = h1; g.ldCb = kHid;
    if ((e = gemm(g, s)) != cudaSuccess) return e;
    g = gdesc();
    g.A = h1; g.a_m = kHid; g.a_k = 1;
    g.B = W + kW2; g.b_k = 1; g.b_n = kHid;
    g.M = n; g.N = kHid; g.K = kHid;
    g.bias = m.params + kB2; g.act = 1; g.Z = z2; g.ldZ = kHid; g.Cb = h2; g.ldCb = kHid;
    if ((e = gemm(g, s)) != cudaSuccess) return e;
    g.A = h2; g.B = W + kW3; g.bias = m.params + kB3; g.Z = z3; g.Cb = h3;
    if ((e = gemm(g, s)) != cudaSuccess) return e;
    g = gdesc();
    g.A = h3; g.a_m = kHid; g.a_k = 1;
    g.B = W + kW4; g.b_k = 1; g.b_n = kHid;
    g.M = n; g.N = kOut; g.K = kHid;
    g.bias = m.params + kB4; g.C = out; g.c_m = kOut; g.c_n = 1;
    return gemm(g, s);
}

// K slices for the weight-gradient products (K = batch rows): ~512 rows each.
constexpr int kMaxSplit = 16;
int split_for(int n)
{
    int sp = (n + 511) / 512;
    return sp < 1 ? 1 : (sp > kMaxSplit ? kMaxSplit : sp);
}

// Backward from dOut (FP32 in m.dOut, BF16 in m.dOutB) to m.grads.
cudaError_t backward(Mlp& m, int n, cudaStream_t s)
{
    const bf16* W = m.pb;
    float* G = m.grads;
    cudaError_t e;
    // dW4 = dOut^T H3 ; db4 = colsum(dOut)
    GemmDesc g = gdesc();
    g.A = m.dOutB; g.a_m = 1; g.a_k = kOut;
    g.B = m.h3; g.b_k = kHid; g.b_n = 1;
    g.M = kOut; g.N = kHid; g.K = n;
    g.C = G + kW4; g.c_m = kHid; g.c_n = 1;
    g.splitK = split_for(n); g.ws = m.ws;
    if ((e = gemm(g, s)) != cudaSuccess) return e;
    if ((e = colsum(m.dOut, n, kOut, kOut, G + kB4, s)) != cudaSuccess) return e;
    // dZ3 = (dOut W4) * silu'(Z3)
    g = gdesc();
    g.A = m.dOutB; g.a_m = kOut; g.a_k = 1;
    g.B = W + kW4; g.b_k = kHid; g.b_n = 1;
    g.M = n; g.N = kHid; g.K = kOut;
    g.dz = m.z3; g.ldz = kHid; g.C = m.dz; g.c_m = kHid; g.c_n = 1; g.Cb = m.dz3; g.ldCb = kHid;
    if ((e = gemm(g, s)) != cudaSuccess) return e;
    // layers 3, 2, 1: dW = dZ^T H_prev, db = colsum(dZ), dZ_prev = (dZ W) * silu'(Z_prev)
    const bf16* dzb[3] = {m.dz3, m.dz2, m.dz1};
    const bf16* hp[3] = {m.h2, m.h1, m.xb};
    const long long wOff[3] = {kW3, kW2, kW1};
    const long long bOff[3] = {kB3, kB2, kB1};
    const int nIn[3] = {kHid, kHid, kIn};
    const float* zPrev[3] = {m.z2, m.z1, nullptr};
    bf16* dzPrev[3] = {m.dz2, m.dz1, nullptr};
    for (int l = 0; l < 3; ++l) {
        g = gdesc();
        g.A = dzb[l]; g.a_m = 1; g.a_k = kHid;
        g.B = hp[l]; g.b_k = nIn[l]; g.b_n = 1;
        g.M = kHid; g.N = nIn[l]; g.K = n;
        g.C = G + wOff[l]; g.c_m = nIn[l]; g.c_n = 1;
        g.splitK = split_for(n); g.ws = m.ws;
        if ((e = gemm(g, s)) != cudaSuccess) return e;
        if ((e = colsum(m.dz, n, kHid, kHid, G + bOff[l], s)) != cudaSuccess) return e;
        if (l == 2) break;
        g = gdesc();
        g.A = dzb[l]; g.a_m = kHid; g.a_k = 1;
        g.B = W + wOff[l]; g.b_k = kHid; g.b_n = 1;
        g.M = n; g.N = kHid; g.K = kHid;
        g.dz = zPrev[l]; g.ldz = kHid; g.C = m.dz; g.c_m = kHid; g.c_n = 1;
        g.Cb = dzPrev[l]; g.ldCb = kHid;
        if ((e = gemm(g, s)) != cudaSuccess) return e;
    }
    return cudaSuccess;
}

template <class T>
cudaError_t alloc(T** p, long long n)
{
    return cudaMalloc((void**)p, (size_t)(n > 0 ? n : 1) * sizeof(T));
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
#define A_(ptr, n) if (e == cudaSuccess) e = alloc(&m->ptr, (n))
    A_(params, kNumParams); A_(grads, kNumParams); A_(m1, kNumParams); A_(m2, kNumParams);
    A_(pb, kNumParams);
    A_(xb, (long long)B * kIn); A_(yl, B); A_(yc, B);
    A_(z1, (long long)B * kHid); A_(z2, (long long)B * kHid); A_(z3, (long long)B * kHid);
    A_(h1, (long long)B * kHid); A_(h2, (long long)B * kHid); A_(h3, (long long)B * kHid);
    A_(out, (long long)B * kOut); A_(dOut, (long long)B * kOut); A_(dOutB, (long long)B * kOut);
    A_(dz, (long long)B * kHid); A_(dz3, (long long)B * kHid); A_(dz2, (long long)B * kHid);
    A_(dz1, (long long)B * kHid);
    A_(loss, 1); A_(step, 1);
    A_(ws, (long long)kMaxSplit * kHid * kHid);
#undef A_
    if (e != cudaSuccess) return report_cuda_error(e, "surrogate network buffers");
    cudaMemset(m->m1, 0, kNumParams * sizeof(float));
    cudaMemset(m->m2, 0, kNumParams * sizeof(float));
    cudaMemset(m->step, 0, sizeof(unsigned long long));
    return CBF_OK;
}

void mlp_free(cbf_mlp* m)
{
    if (m->exec) cudaGraphExecDestroy(m->exec);
    if (m->graph) cudaGraphDestroy(m->graph);
    void* ptrs[] = {m->params, m->grads, m->m1, m->m2, m->pb, m->xb, m->yl, m->yc, m->z1, m->z2,
                    m->z3, m->h1, m->h2, m->h3, m->out, m->dOut, m->dOutB, m->dz, m->dz3,
                    m->dz2, m->dz1, m->loss, m->ws, m->step, m->pxb, m->ph1, m->ph2, m->ph3, m->pout,
                    m->wpack, m->tcErr};
    for (void* p : ptrs) cudaFree(p);
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
            to_bf16_kernel<<<b, t>>>(m->params, m->pb, kNumParams);
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

// One forward + backward on host data (n <= batch rows); for gradient checks.
cbf_status cbf_mlp_forward_backward(cbf_mlp* m, const float* hx, const float* hyl, const int32_t* hyc,
                                    int32_t n, float wLle, float* hloss, float* hgrads, float* hout)
{
    if (!m || !hx || !hyl || !hyc || n < 1 || n > m->B)
        return report_error(CBF_ERR_INVALID_ARG, "bad batch");
    std::vector<bf16> xb((size_t)n * kIn);
    for (long long i = 0; i < (long long)n * kIn; ++i) xb[i] = __float2bfloat16_rn(hx[i]);
    cudaError_t e = cudaMemcpy(m->xb, xb.data(), xb.size() * sizeof(bf16), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(m->yl, hyl, (size_t)n * sizeof(float), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(m->yc, hyc, (size_t)n * sizeof(int), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(m->loss, 0, sizeof(float));
    if (e == cudaSuccess) e = forward(*m, n, m->xb, m->out, m->z1, m->z2, m->z3, m->h1, m->h2, m->h3, 0);
    if (e == cudaSuccess)
        e = launch1d(n, 0, [&](unsigned b, int t) {
            loss_kernel<<<b, t>>>(m->out, m->yl, m->yc, n, wLle, m->dOut, m->dOutB, m->loss);
        });
    if (e == cudaSuccess) e = backward(*m, n, 0);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
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
        m->gW != wLle || m->gSeed != m->seed) {
        if (m->exec) cudaGraphExecDestroy(m->exec);
        if (m->graph) cudaGraphDestroy(m->graph);
        m->exec = nullptr;
        m->graph = nullptr;
        e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) return report_cuda_error(e, "begin capture of the training step");
        cudaError_t ce = launch1d(B, s, [&](unsigned b, int t) {
            gather_kernel<<<b, t, 0, s>>>(dX, dYl, (const int*)dYc, N, B, m->step, m->seed, m->xb,
                                          m->yl, m->yc);
        });
        if (ce == cudaSuccess) ce = forward(*m, B, m->xb, m->out, m->z1, m->z2, m->z3, m->h1, m->h2, m->h3, s);
        if (ce == cudaSuccess)
            ce = launch1d(B, s, [&](unsigned b, int t) {
                loss_kernel<<<b, t, 0, s>>>(m->out, m->yl, m->yc, B, wLle, m->dOut, m->dOutB, m->loss);
            });
        if (ce == cudaSuccess) ce = backward(*m, B, s);
        if (ce == cudaSuccess)
            ce = launch1d(kNumParams, s, [&](unsigned b, int t) {
                adam_kernel<<<b, t, 0, s>>>(m->params, m->grads, m->m1, m->m2, m->pb, kNumParams, lr,
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
    if (e != cudaSuccess) return report_cuda_error(e, "training");
    return CBF_OK;
}

// Predictions for N feature rows (device X [N x 4] FP32): LLE (de-normalised
// with lleMean/lleStd), class, softmax confidence.  Runs in chunks of `batch`
// rows through the training buffers.
cbf_status cbf_mlp_predict(cbf_mlp* m, const float* dX, int64_t N, float lleMean, float lleStd,
                           float* dLle, int32_t* dCls, float* dConf, void* stream)
{
    if (!m || !dX || N < 0) return report_error(CBF_ERR_INVALID_ARG, "bad prediction arguments");
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e = cudaSuccess;
    if ((e = pred_workspace(m)) != cudaSuccess) return report_cuda_error(e, "prediction workspace");
    for (long long r0 = 0; r0 < N && e == cudaSuccess; r0 += kPredRows) {
        const int n = (int)((N - r0) < kPredRows ? (N - r0) : kPredRows);
        e = launch1d((long long)n * kIn, s, [&](unsigned b, int t) {
            to_bf16_kernel<<<b, t, 0, s>>>(dX + r0 * kIn, m->pxb, (long long)n * kIn);
        });
        if (e == cudaSuccess)
            e = forward(*m, n, m->pxb, m->pout, nullptr, nullptr, nullptr, m->ph1, m->ph2, m->ph3, s);
        if (e == cudaSuccess)
            e = launch1d(n, s, [&](unsigned b, int t) {
                head_kernel<<<b, t, 0, s>>>(m->pout, n, lleMean, lleStd, dLle ? dLle + r0 : nullptr,
                                            dCls ? (int*)dCls + r0 : nullptr, dConf ? dConf + r0 : nullptr);
            });
    }
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
    mlp_predict_tc_kernel<<<grid, kTcThreads, kTcSmem, s>>>(f, nPoints, m->wpack, m->params, lleMean, lleStd, lle,
                                                            cls, conf, m->tcErr);
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
