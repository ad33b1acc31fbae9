// Matrix products of the surrogate network's training step (and of the
// prediction of explicit feature rows) on the 5th-generation tensor cores.
// Included by mlp.cu after mlp_tc.cuh, inside its anonymous namespace (uses its
// descriptor, mbarrier and tensor-memory helpers, silu and silu_grad).
//
// One kernel form computes every product: a 128 x BN tile of
//     D = A[M x K] * B[N x K]^T
// with both operands K-contiguous BF16 matrices in global memory.  The
// transposed operands that backpropagation needs are written as extra outputs
// by the kernels that produce them -- H^T and dZ^T by this kernel's epilogues,
// X^T by the minibatch gather, dOut^T by the loss, W^T by the Adam step -- so no
// product ever reads a matrix across its rows.
//
// Operands reach shared memory by TMA (cp.async.bulk.tensor, 4-D tensor maps)
// directly in the UMMA K-major no-swizzle core-matrix layout.  The tensor map of
// a row-major R x C BF16 matrix with row pitch ld elements is the 4-D view
//     (k_in 8, r_in 8, r_grp R/8, k_grp C/8),  byte strides (2, 2 ld, 16 ld, 16)
// and its box (8, 8, rows/8, kc/8) lands in shared memory at
//     k_in*2 + r_in*16 + r_grp*128 + k_grp*(rows*16)  bytes,
// i.e. element (r, k) of the tile at tc_off(rows, r, k): leading-dimension byte
// offset rows*16 (between 8-column groups), stride-dimension byte offset 128
// (between 8-row groups), as in mlp_tc.cuh.  The innermost coordinate of every
// copy is 0 (16-byte aligned).  Every tensor map covers at least 128 KiB: the
// buffers are allocated at least that large.
//
// CTA: 256 threads.  Thread 0 issues the copies of up to four K chunks (one
// mbarrier each), then for each chunk, once it has landed, the KC/16
// tcgen05.mma.cta_group::1.kind::f16 instructions (M 128, N BN) into an FP32
// accumulator of BN tensor-memory columns, and commits them to a "done"
// mbarrier; longer K slices run in passes of four chunks.  The eight warps then
// read the accumulator (tcgen05.ld.32x32b.x32, warp w: lanes 32(w%4).., every
// other 32-column chunk) and apply the epilogue:
//   kEpiHidden  z = acc + bias -> Z (FP32), h = SiLU(z) -> H (BF16) and H^T
//   kEpiOut     acc + bias -> C (FP32), the columns n < Nv
//   kEpiDgrad   d = acc * SiLU'(zp) -> C (FP32), H (BF16), H^T (BF16)
//   kEpiWgrad   acc -> C, or the K slice's partial into ws (split K; the
//               slices are added in order by splitk_reduce_kernel)
// Rows m >= Mv of a tile write zeros into H^T, so that a later product whose K
// runs over the padded batch adds nothing for them.  Every mbarrier wait is
// bounded: a wait that runs out drains the copies and products in flight (again
// bounded), sets the error flag and frees the tensor memory.  (mlp.cu includes
// <cuda.h> for the tensor-map types.)

constexpr int kGtM = 128;
constexpr int kGtThreads = 256;
constexpr int kGtStages = 4;
constexpr size_t kGtMaxSmem = (size_t)kGtStages * (kGtM + 256) * 64 * 2 + 128;

enum { kEpiHidden = 0, kEpiOut = 1, kEpiDgrad = 2, kEpiWgrad = 3 };

struct TcGemm {
    int M, N, K;     // rows computed (tiles of 128), columns (a multiple of BN), reduction length
    int BN, KC;      // column tile (16..256, a multiple of 16), K chunk (16, 32 or 64)
    int kSlice;      // K of one split (a multiple of KC); gridDim.z = ceil(K / kSlice)
    int Mv, Nv;      // rows and columns of the result that exist
    int mode;
    const float* bias;
    const float* zp;  // kEpiDgrad: pre-activation whose SiLU derivative scales the product
    long long ldzp;
    float* Z;         // kEpiHidden: pre-activation (after bias), row-major
    long long ldZ;
    float* C;         // FP32 result, row-major
    long long ldc;
    bf16* Hb;         // BF16 result, row-major
    long long ldh;
    bf16* HT;         // BF16 result transposed: HT[n * ldht + m]
    long long ldht;
    float* ws;        // kEpiWgrad with splits: ws[(z * Mv + m) * Nv + n]
    int* err;
};

// 4-D tiled tensor copy global -> shared completing on `bar`.
__device__ __forceinline__ void tma_load4(uint32_t dst, const CUtensorMap* map, int c0, int c1, int c2, int c3,
                                          uint32_t bar)
{
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
        "[%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(bar)
        : "memory");
}

__device__ __forceinline__ void store_f32x32(float* p, const float (&v)[32])
{
#pragma unroll
    for (int i = 0; i < 8; ++i)
        reinterpret_cast<float4*>(p)[i] = make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
}

__device__ __forceinline__ void store_bf16x32(bf16* p, const float (&v)[32])
{
#pragma unroll
    for (int i = 0; i < 4; ++i)
        reinterpret_cast<uint4*>(p)[i] =
            make_uint4(pack_bf16x2(v[8 * i], v[8 * i + 1]), pack_bf16x2(v[8 * i + 2], v[8 * i + 3]),
                       pack_bf16x2(v[8 * i + 4], v[8 * i + 5]), pack_bf16x2(v[8 * i + 6], v[8 * i + 7]));
}

__global__ void __launch_bounds__(kGtThreads, 1)
    gemm_tc_kernel(const __grid_constant__ CUtensorMap ta, const __grid_constant__ CUtensorMap tb, const TcGemm g)
{
    extern __shared__ __align__(1024) unsigned char gsm[];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.x * kGtM, n0 = blockIdx.y * g.BN;
    const int kBeg = blockIdx.z * g.kSlice;
    const int kEnd = min(g.K, kBeg + g.kSlice);
    const int nch = (kEnd - kBeg) / g.KC;
    const int S = nch < kGtStages ? nch : kGtStages;
    const uint32_t aBytes = (uint32_t)(kGtM * g.KC * 2), stBytes = aBytes + (uint32_t)(g.BN * g.KC * 2);
    uint64_t* bars = reinterpret_cast<uint64_t*>(gsm + (size_t)kGtStages * stBytes);  // full[4], done
    uint32_t* slot = reinterpret_cast<uint32_t*>(bars + kGtStages + 1);
    int* flag = reinterpret_cast<int*>(slot + 1);
    const uint32_t base = smem_u32(gsm);
    const uint32_t doneBar = smem_u32(&bars[kGtStages]);
    const uint32_t cols = g.BN <= 32 ? 32u : (g.BN <= 64 ? 64u : (g.BN <= 128 ? 128u : 256u));

    if (tid == 0) {
        for (int i = 0; i <= kGtStages; ++i) mbar_init(smem_u32(&bars[i]), 1);
        *flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)),
                     "r"(cols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *slot;

    if (tid == 0 && nch > 0) {
        const uint32_t idesc = tc_idesc(kGtM, g.BN);
        bool ok = true;
        int pass = 0;
        for (int c0 = 0; c0 < nch; c0 += S, ++pass) {
            const int cn = min(S, nch - c0);
            const uint32_t par = (uint32_t)(pass & 1);
            for (int j = 0; j < cn; ++j) {
                const uint32_t fb = smem_u32(&bars[j]);
                const int kg = (kBeg + (c0 + j) * g.KC) >> 3;
                mbar_expect_tx(fb, stBytes);
                tma_load4(base + (uint32_t)j * stBytes, &ta, 0, 0, m0 >> 3, kg, fb);
                tma_load4(base + (uint32_t)j * stBytes + aBytes, &tb, 0, 0, n0 >> 3, kg, fb);
            }
            int j = 0;
            for (; j < cn; ++j) {
                if (!mbar_wait(smem_u32(&bars[j]), par)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                const uint32_t aAddr = base + (uint32_t)j * stBytes, bAddr = aAddr + aBytes;
                for (int kk = 0; kk < g.KC / 16; ++kk) {
                    const uint64_t a = tc_desc(aAddr + (uint32_t)kk * 2u * (kGtM * 16), kGtM * 16, 128);
                    const uint64_t b = tc_desc(bAddr + (uint32_t)kk * 2u * (uint32_t)(g.BN * 16),
                                               (uint32_t)(g.BN * 16), 128);
                    tc_mma(tmem, a, b, idesc, (c0 + j > 0 || kk > 0) ? 1u : 0u);
                }
            }
            // on a failed wait: let the copies still in flight land (bounded)
            if (!ok)
                for (int r = j; r < cn; ++r) mbar_wait(smem_u32(&bars[r]), par);
            tc_commit(doneBar);
            if (!mbar_wait(doneBar, par)) ok = false;  // the products have read every stage
            if (!ok) break;
        }
        if (!ok) *flag = 1;
    }
    __syncthreads();
    tc_fence_after();
    const bool bad = *flag != 0;

    if (!bad && nch > 0) {
        const int q = warp & 3, half = warp >> 2;
        const int row = m0 + 32 * q + lane;
        const bool rv = row < g.Mv;
        const uint32_t lb = tmem + ((uint32_t)(32 * q) << 16);
        const int nChunks = (g.BN + 31) / 32;
        for (int ch = half; ch < nChunks; ch += 2) {
            float v[32];
            tmem_ld32(lb + (uint32_t)(ch * 32), v);
            const int nb = n0 + ch * 32;
            if (g.mode == kEpiHidden) {
#pragma unroll
                for (int j = 0; j < 32; ++j) v[j] += g.bias[nb + j];
                if (rv && g.Z) store_f32x32(g.Z + row * g.ldZ + nb, v);
#pragma unroll
                for (int j = 0; j < 32; ++j) v[j] = silu(v[j]);
                if (rv && g.Hb) store_bf16x32(g.Hb + row * g.ldh + nb, v);
                if (g.HT) {
#pragma unroll
                    for (int j = 0; j < 32; ++j)
                        g.HT[(long long)(nb + j) * g.ldht + row] = __float2bfloat16_rn(rv ? v[j] : 0.0f);
                }
            } else if (g.mode == kEpiDgrad) {
                if (rv) {
                    const float4* z4 = reinterpret_cast<const float4*>(g.zp + row * g.ldzp + nb);
#pragma unroll
                    for (int i = 0; i < 8; ++i) {
                        const float4 z = z4[i];
                        v[4 * i] *= silu_grad(z.x);
                        v[4 * i + 1] *= silu_grad(z.y);
                        v[4 * i + 2] *= silu_grad(z.z);
                        v[4 * i + 3] *= silu_grad(z.w);
                    }
                    if (g.C) store_f32x32(g.C + row * g.ldc + nb, v);
                    if (g.Hb) store_bf16x32(g.Hb + row * g.ldh + nb, v);
                }
                if (g.HT) {
#pragma unroll
                    for (int j = 0; j < 32; ++j)
                        g.HT[(long long)(nb + j) * g.ldht + row] = __float2bfloat16_rn(rv ? v[j] : 0.0f);
                }
            } else if (g.mode == kEpiOut) {
                if (rv)
#pragma unroll
                    for (int j = 0; j < 32; ++j)
                        if (nb + j < g.Nv) g.C[row * g.ldc + nb + j] = v[j] + g.bias[nb + j];
            } else if (rv) {  // kEpiWgrad
                float* dst = gridDim.z > 1 ? g.ws + ((long long)blockIdx.z * g.Mv + row) * g.Nv
                                           : g.C + row * g.ldc;
                const long long ld = gridDim.z > 1 ? g.Nv : g.ldc;
                if (nb + 32 <= g.Nv && (ld & 3) == 0 && ((uintptr_t)dst & 15) == 0) {
                    store_f32x32(dst + nb, v);
                } else {
#pragma unroll
                    for (int j = 0; j < 32; ++j)
                        if (nb + j < g.Nv) dst[nb + j] = v[j];
                }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(cols) : "memory");
    if (bad && tid == 0) atomicExch(g.err, 1);
}

// ---- host side -------------------------------------------------------------

typedef CUresult (*TensorMapEncodeFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                      const cuuint64_t*, const cuuint32_t*, const cuuint32_t*,
                                      CUtensorMapInterleave, CUtensorMapSwizzle, CUtensorMapL2promotion,
                                      CUtensorMapFloatOOBfill);

// The driver's cuTensorMapEncodeTiled, looked up once through the runtime (no
// link against libcuda).
cudaError_t tensor_map_encoder(TensorMapEncodeFn* out)
{
    static TensorMapEncodeFn fn = nullptr;
    static cudaError_t status = cudaSuccess;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        status = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q);
        if (status == cudaSuccess && (q != cudaDriverEntryPointSuccess || !p)) status = cudaErrorNotSupported;
        fn = reinterpret_cast<TensorMapEncodeFn>(p);
    });
    *out = fn;
    return status;
}

// Tensor map of the row-major R x Cc BF16 matrix at p (row pitch ld elements)
// for operand tiles of `rows` x `kc` (see the layout at the top of this file).
cudaError_t operand_map(CUtensorMap* map, const bf16* p, long long R, long long Cc, long long ld, int rows, int kc)
{
    if (!p || R % 8 || Cc % 8 || ld % 8 || rows % 8 || kc % 8 || rows > R || kc > Cc || Cc > ld ||
        ((uintptr_t)p & 15) || R * ld * 2 < (128ll << 10) || rows / 8 > 256 || kc / 8 > 256)
        return cudaErrorInvalidValue;
    TensorMapEncodeFn enc = nullptr;
    cudaError_t e = tensor_map_encoder(&enc);
    if (e != cudaSuccess) return e;
    const cuuint64_t dims[4] = {8, 8, (cuuint64_t)(R / 8), (cuuint64_t)(Cc / 8)};
    const cuuint64_t strides[3] = {(cuuint64_t)ld * 2, (cuuint64_t)ld * 16, 16};
    const cuuint32_t box[4] = {8, 8, (cuuint32_t)(rows / 8), (cuuint32_t)(kc / 8)};
    const cuuint32_t es[4] = {1, 1, 1, 1};
    const CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<bf16*>(p), dims, strides, box, es,
                           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                           CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

// One product: A through `ta` (128-row tiles, KC-wide), B through `tb` (BN-row
// tiles, KC-wide); split-K partials are added in slice order afterwards.
cudaError_t gemm_tc(const CUtensorMap& ta, const CUtensorMap& tb, const TcGemm& g, cudaStream_t s)
{
    if (g.M <= 0 || g.Mv <= 0) return cudaSuccess;
    if (g.BN < 16 || g.BN > 256 || g.BN % 16 || g.N % g.BN || (g.KC != 16 && g.KC != 32 && g.KC != 64) ||
        g.K <= 0 || g.K % g.KC || g.kSlice <= 0 || g.kSlice % g.KC || g.Nv > g.N ||
        ((g.mode == kEpiHidden || g.mode == kEpiDgrad) && g.BN % 32))
        return cudaErrorInvalidValue;
    const int splits = (g.K + g.kSlice - 1) / g.kSlice;
    if (splits > 1 && (g.mode != kEpiWgrad || !g.ws)) return cudaErrorInvalidValue;
    const dim3 grid((unsigned)((g.M + kGtM - 1) / kGtM), (unsigned)(g.N / g.BN), (unsigned)splits);
    const size_t smem = (size_t)kGtStages * (kGtM + g.BN) * g.KC * 2 + 64;
    gemm_tc_kernel<<<grid, kGtThreads, smem, s>>>(ta, tb, g);
    note_launch();
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess || splits == 1) return e;
    const long long MN = (long long)g.Mv * g.Nv;
    splitk_reduce_kernel<<<(unsigned)((MN + 255) / 256), 256, 0, s>>>(g.ws, splits, g.Mv, g.Nv, g.C, g.ldc, 1);
    note_launch();
    return cudaGetLastError();
}

TcGemm tc_gemm(int mode, int* err)
{
    TcGemm g;
    memset(&g, 0, sizeof(g));
    g.mode = mode;
    g.err = err;
    return g;
}
