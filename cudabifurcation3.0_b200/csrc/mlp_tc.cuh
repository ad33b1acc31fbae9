// Grid prediction of the surrogate network on the 5th-generation tensor cores:
// tcgen05.mma (BF16 x BF16 -> FP32, M = 128) with the accumulator in tensor
// memory, operands in shared memory, weights brought in by bulk async copies.
// Included by mlp.cu inside its anonymous namespace (uses its constants,
// point_features, encode8, pack_bf16x2 and silu).
//
// One persistent CTA per SM (512 threads, 192 KB of shared memory) takes tiles
// of 128 grid points:
//   features (4 inputs and their 124 Fourier terms, K = 128) -> A buffer
//   layer 1: 8 MMAs (K 128, N 256) | layers 2, 3: 16 MMAs (K 256, N 256)
//   | layer 4: 16 MMAs (K 256, N 32: the 17 outputs and zero rows)
// Between layers the accumulator (128 lanes x 256 FP32 columns of tensor
// memory) is read with tcgen05.ld, bias + SiLU applied, rounded to BF16 and
// written back into the A buffer as the next layer's operand; the next
// layer's weights are copied into the B buffer meanwhile.  The last epilogue
// is the prediction head (LLE, argmax class, softmax confidence).
//
// Shared-memory operand layout (K-major, no swizzle): 8 x 16-byte "core
// matrices" (8 rows, 8 consecutive k), element (r, k) of an R-row operand at
//   (k / 8) * (R * 16) + (r / 8) * 128 + (r % 8) * 16 + (k % 8) * 2  bytes,
// i.e. leading-dimension byte offset (between the two 8-k halves of one
// K = 16 MMA) R * 16, stride-dimension byte offset (between 8-row groups) 128.
// The weights are packed once per call into exactly this layout in global
// memory, so each layer's copy is a plain contiguous bulk copy.

constexpr int kTcM = 128;        // grid points per tile (MMA M, tensor-memory lanes)
constexpr int kTcThreads = 512;  // 16 warps: four per tensor-memory lane quarter
constexpr int kTcCols = 256;     // tensor-memory columns allocated (FP32 accumulator N = 256)
constexpr int kTcN4 = 32;        // layer-4 MMA N: 17 outputs padded with zero rows
constexpr uint32_t kTcABytes = kTcM * kHid * 2;      // 65536
constexpr uint32_t kTcBBytes = kHid * kHid * 2;      // 131072
constexpr uint32_t kTcW1Bytes = kHid * kIn * 2;      // 65536
constexpr uint32_t kTcW4Bytes = kTcN4 * kHid * 2;    // 16384
constexpr uint32_t kTcPackBytes = kTcW1Bytes + 2 * kTcBBytes + kTcW4Bytes;
constexpr size_t kTcSmem = kTcABytes + kTcBBytes + 64;
constexpr long long kTcSpin = 1ll << 22;  // polls of an mbarrier before giving up (~0.3 s)

// Byte offset of element (r, k) in an R-row K-major core-matrix operand.
__host__ __device__ constexpr uint32_t tc_off(int R, int r, int k)
{
    return (uint32_t)((k >> 3) * (R * 16) + (r >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor: start, LBO, SBO in 16-byte units, version 1
// (sm_100), no swizzle.
__device__ __forceinline__ uint64_t tc_desc(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
    return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both
// K-major, N >> 3 at bit 17, M >> 4 at bit 24.
__host__ __device__ constexpr uint32_t tc_idesc(int M, int N)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void tc_mma(uint32_t tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
        :
        : "r"(tmem), "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
        : "memory");
}

__device__ __forceinline__ void tc_commit(uint32_t bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait for the completion of phase `parity`; false if it never came.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity)
{
    for (long long it = 0; it < kTcSpin; ++it) {
        if (mbar_try_wait(bar, parity)) return true;
        if (it > 64) __nanosleep(64);
    }
    return false;
}

// Contiguous global -> shared bulk copy completing on `bar` (16-byte aligned,
// size a multiple of 16).
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}

// 32 consecutive FP32 columns of this thread's tensor-memory lane.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32])
{
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
        "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr)
        : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int j = 0; j < 32; ++j) v[j] = __uint_as_float(r[j]);
}


// The BF16 weights (flat layout of the parameter buffer) in the shared-memory
// operand layout: W1 (256 x 4, K padded to 16), W2, W3 (256 x 256), W4 (17 x
// 256, rows padded to 32), one 2-byte element per thread.
__global__ void tc_pack_kernel(const bf16* __restrict__ pb, bf16* __restrict__ out)
{
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= kTcPackBytes / 2) return;
    uint32_t o = (uint32_t)e * 2;
    int R, K;
    long long src;
    if (o < kTcW1Bytes) {
        R = kHid; K = kIn; src = kW1;
    } else if ((o -= kTcW1Bytes) < kTcBBytes) {
        R = kHid; K = kHid; src = kW2;
    } else if ((o -= kTcBBytes) < kTcBBytes) {
        R = kHid; K = kHid; src = kW3;
    } else {
        o -= kTcBBytes;
        R = kTcN4; K = kHid; src = kW4;
    }
    const int kc = (int)(o / (uint32_t)(R * 16));
    const uint32_t rem = o % (uint32_t)(R * 16);
    const int r = (int)(rem / 128) * 8 + (int)((rem % 128) / 16);
    const int k = kc * 8 + (int)((rem % 16) / 2);
    const int rows = (src == kW4) ? kOut : kHid;
    out[e] = (r < rows && k < K) ? pb[src + (long long)r * K + k] : __float2bfloat16_rn(0.0f);
}

// Issue the MMAs of one layer (one thread) once its weights have arrived.
__device__ __forceinline__ void tc_issue(uint32_t tmem, uint32_t aAddr, uint32_t bAddr, int slices, uint32_t lboB,
                                         uint32_t idesc)
{
    for (int sl = 0; sl < slices; ++sl) {
        const uint64_t a = tc_desc(aAddr + (uint32_t)sl * 2u * (kTcM * 16), kTcM * 16, 128);
        const uint64_t b = tc_desc(bAddr + (uint32_t)sl * 2u * lboB, lboB, 128);
        tc_mma(tmem, a, b, idesc, sl > 0 ? 1u : 0u);
    }
}

__global__ void __launch_bounds__(kTcThreads, 1)
    mlp_predict_tc_kernel(const FeatureSpec f, long long nPoints, float fs, const unsigned char* __restrict__ wpack,
                          const float* __restrict__ params, float lleMean, float lleStd, double* __restrict__ lle,
                          int* __restrict__ cls, float* __restrict__ conf, int* __restrict__ err)
{
    extern __shared__ __align__(1024) unsigned char tsm[];
    unsigned char* A = tsm;
    uint64_t* bars = reinterpret_cast<uint64_t*>(tsm + kTcABytes + kTcBBytes);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(bars + 2);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t aAddr = smem_u32(tsm), bAddr = smem_u32(tsm + kTcABytes);
    const uint32_t wbar = smem_u32(&bars[0]), mbar = smem_u32(&bars[1]);

    if (tid == 0) {
        mbar_init(wbar, 1);
        mbar_init(mbar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                     "r"(kTcCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;

    const int q = warp & 3;      // tensor-memory lane quarter: tile rows 32q .. 32q+31
    const int part = warp >> 2;  // column quarter (64 columns) of the hidden-layer epilogues
    const int row = 32 * q + lane;
    const uint32_t laneBase = tmem + ((uint32_t)(32 * q) << 16);
    const unsigned char* wNext[4] = {wpack, wpack + kTcW1Bytes, wpack + kTcW1Bytes + kTcBBytes,
                                     wpack + kTcW1Bytes + 2 * kTcBBytes};
    const uint32_t wBytes[4] = {kTcW1Bytes, kTcBBytes, kTcBBytes, kTcW4Bytes};
    const float* bias[3] = {params + kB1, params + kB2, params + kB3};
    uint32_t wph = 0, mph = 0;
    bool bad = false;

    // thread 0: bring layer L's weights into the B buffer (free by now)
    auto fetch = [&](int L) {
        if (tid != 0) return;
        mbar_expect_tx(wbar, wBytes[L]);
        for (uint32_t o = 0; o < wBytes[L]; o += 16384u) {
            const uint32_t b = wBytes[L] - o < 16384u ? wBytes[L] - o : 16384u;
            bulk_g2s(bAddr + o, wNext[L] + o, b, wbar);
        }
    };
    // layer L's MMAs once its weights are in; every thread then waits for them
    auto layer = [&](int L) -> bool {
        int fail = 0;
        if (tid == 0) {
            if (mbar_wait(wbar, wph)) {
                tc_fence_after();
                if (L == 0) tc_issue(tmem, aAddr, bAddr, kIn / 16, kHid * 16, tc_idesc(kTcM, kHid));
                else if (L < 3) tc_issue(tmem, aAddr, bAddr, kHid / 16, kHid * 16, tc_idesc(kTcM, kHid));
                else tc_issue(tmem, aAddr, bAddr, kHid / 16, kTcN4 * 16, tc_idesc(kTcM, kTcN4));
                tc_commit(mbar);
            } else {
                fail = 1;
            }
        }
        wph ^= 1;
        if (__syncthreads_or(fail)) return false;
        const bool ok = mbar_wait(mbar, mph);
        mph ^= 1;
        tc_fence_after();
        return !__syncthreads_or(!ok);
    };
    // all threads: make this thread's tensor-memory reads and A writes visible
    // to the next MMAs
    auto handoff = [&]() {
        fence_async_smem();
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
    };

    const long long nTiles = (nPoints + kTcM - 1) / kTcM;
    for (long long tile = blockIdx.x; tile < nTiles && !bad; tile += gridDim.x) {
        const long long r0 = tile * kTcM;
        fetch(0);
        {
            // four threads per point, each encoding 4 of its 16 groups of 8 inputs
            const int pt = tid >> 2, part = tid & 3;
            float x[kRaw] = {0.f, 0.f, 0.f, 0.f};
            const bool live = r0 + pt < nPoints;
            if (live) point_features(f, r0 + pt, x);
            for (int j = part; j < kIn / 8; j += 4) {
                float e[8];
                encode8(x, j, fs, e);
                *reinterpret_cast<uint4*>(A + tc_off(kTcM, pt, 8 * j)) =
                    live ? make_uint4(pack_bf16x2(e[0], e[1]), pack_bf16x2(e[2], e[3]), pack_bf16x2(e[4], e[5]),
                                      pack_bf16x2(e[6], e[7]))
                         : make_uint4(0u, 0u, 0u, 0u);
            }
        }
        handoff();
        for (int L = 0; L < 4 && !bad; ++L) {
            if (!layer(L)) {
                bad = true;
                break;
            }
            if (L < 3) {
                fetch(L + 1);
                // bias + SiLU of 64 columns of this thread's row, BF16 into A
                const float* bL = bias[L];
                for (int c = 0; c < 2; ++c) {
                    const int col0 = part * 64 + c * 32;
                    float v[32];
                    tmem_ld32(laneBase + (uint32_t)col0, v);
                    uint32_t pk[16];
#pragma unroll
                    for (int j = 0; j < 32; j += 2)
                        pk[j / 2] = pack_bf16x2(silu(v[j] + bL[col0 + j]), silu(v[j + 1] + bL[col0 + j + 1]));
#pragma unroll
                    for (int i = 0; i < 4; ++i)
                        *reinterpret_cast<uint4*>(A + tc_off(kTcM, row, col0 + 8 * i)) =
                            make_uint4(pk[4 * i], pk[4 * i + 1], pk[4 * i + 2], pk[4 * i + 3]);
                }
            } else if (part == 0) {
                // prediction head, as head_kernel
                float v[32];
                tmem_ld32(laneBase, v);
                const long long r = r0 + row;
                if (r < nPoints) {
                    const float* b4 = params + kB4;
                    float o[kOut];
#pragma unroll
                    for (int j = 0; j < kOut; ++j) o[j] = v[j] + b4[j];
                    int best = 0;
                    float mx = o[1];
#pragma unroll
                    for (int c = 1; c < kClasses; ++c)
                        if (o[1 + c] > mx) {
                            mx = o[1 + c];
                            best = c;
                        }
                    float sum = 0.f;
#pragma unroll
                    for (int c = 0; c < kClasses; ++c) sum += __expf(o[1 + c] - mx);
                    lle[r] = (double)(o[0] * lleStd + lleMean);
                    cls[r] = best;
                    conf[r] = 1.0f / sum;
                }
            }
            handoff();
        }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTcCols) : "memory");
    if (bad && tid == 0) atomicExch(err, 1);
}
