// Kernels of the learned period-proposal network (sm_100a).  No counterpart in
// the reference: the network ranks log-period windows of the full BLS grid so
// that the exact search can be restricted to them.
//
//   * pn_gemm_kernel<BN>: D[M, N] = A[M, K] . B[N, K]^T, bf16 operands (both
//     K-major), fp32 accumulation in tensor memory.  One CTA per 128 x BN output
//     tile (grid.z splits K): thread 0 streams 128 x 64 and BN x 64 tiles of A
//     and B into a four-stage shared-memory ring with TMA (128-byte swizzle,
//     each CTA loading its own tiles), thread 32 issues tcgen05.mma (M = 128,
//     N = BN, K = 16 per instruction) as each stage lands and returns the stage
//     to the producer with tcgen05.commit, and the four warps read the
//     accumulator back with tcgen05.ld (warp w owns rows 32w..32w+31) for a
//     fused epilogue: bias, ReLU, a ReLU-derivative mask, bf16 or fp32 store
//     (optionally transposed), or fp32 atomic accumulation for split-K.  Every
//     wait on an mbarrier is bounded by the global timer; a wait that runs out
//     sets the error flag, the CTA skips its stores, frees its tensor memory and
//     returns.
//   * the network's data movers and small steps: time binning of the curves,
//     im2col / col2im for the stride-2 convolutions, transposes, bias
//     gradients, softmax cross-entropy, Adam, and the top-k window selection.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <mutex>

#include "../../include/bls_proposal.h"

namespace blsb200 {
namespace pn {
namespace {

constexpr int kBM = 128;
constexpr int kBK = 64;                 // bf16: one 128-byte swizzle row
constexpr int kStages = 4;
constexpr int kGemmThreads = 128;
constexpr unsigned long long kWaitNs = 2000000000ull;     // 2 s per wait

struct GemmArgs {
    int M, N, K;
    int kb_per_split;
    void* out;
    long long ldo;
    int out_mode;           // PN_OUT_BF16 / PN_OUT_F32 / PN_OUT_F32_ADD
    int transpose_out;      // element (m, n) at out[n * ldo + m]
    const float* bias;      // per n, or null
    int relu;
    const __nv_bfloat16* mask;      // multiply by (mask[m, n] > 0), ld = ldo, or null
    int* error_flag;
};

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

// Wait for the phase of `parity` to complete, for at most kWaitNs.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = global_ns();
    while (!mbar_try_wait(bar, parity))
        if (global_ns() - t0 > kWaitNs) return false;
    return true;
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* tm, int x, int y,
                                            uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(tm)), "r"(x), "r"(y), "r"(bar)
        : "memory");
}

// Shared-memory matrix descriptor of a K-major tile stored as rows of 128 bytes
// with the 128-byte swizzle (what TMA writes with CU_TENSOR_MAP_SWIZZLE_128B):
// start address >> 4, leading byte offset 16 B (unused for this layout), stride
// byte offset 1024 B between 8-row groups, descriptor version 1, layout 2.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t addr) {
    return (uint64_t)((addr & 0x3FFFFu) >> 4) | ((uint64_t)1 << 16) |
           ((uint64_t)(1024 >> 4) << 32) | ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

// Instruction descriptor of kind::f16: D fp32, A and B bf16, both K-major, M x N.
__host__ __device__ constexpr uint32_t bf16_idesc(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) |
           ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b,
                                          uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}" ::"r"(tmem_d),
        "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ void umma_commit(uint32_t bar) {
    asm volatile(
        "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
        : "memory");
}

__device__ __forceinline__ void tc_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// 16 consecutive fp32 columns of the accumulator for this warp's 32 rows.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10,"
        " %11, %12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
          "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int j = 0; j < 16; ++j) v[j] = __uint_as_float(r[j]);
}

template <int BN>
__global__ void __launch_bounds__(kGemmThreads, 1)
    pn_gemm_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                   const GemmArgs g) {
    constexpr uint32_t kABytes = kBM * kBK * 2;
    constexpr uint32_t kBBytes = BN * kBK * 2;
    extern __shared__ uint8_t dsm_raw[];
    __shared__ __align__(8) uint64_t full_bar[kStages];
    __shared__ __align__(8) uint64_t empty_bar[kStages];
    __shared__ __align__(8) uint64_t done_bar;
    __shared__ uint32_t tmem_slot;
    __shared__ int abort_s;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nk_total = (g.K + kBK - 1) / kBK;
    const int kb0 = blockIdx.z * g.kb_per_split;
    const int nk = min(g.kb_per_split, nk_total - kb0);
    if (nk <= 0) return;                        // the same for every thread of the CTA
    const int m0 = blockIdx.x * kBM, n0 = blockIdx.y * BN;

    // tiles on 1024-byte boundaries (the swizzle atom)
    const uint32_t raw = (uint32_t)__cvta_generic_to_shared(dsm_raw);
    const uint32_t sA = (raw + 1023u) & ~1023u;
    const uint32_t sB = sA + kStages * kABytes;
    const uint32_t fb = (uint32_t)__cvta_generic_to_shared(full_bar);
    const uint32_t eb = (uint32_t)__cvta_generic_to_shared(empty_bar);
    const uint32_t db = (uint32_t)__cvta_generic_to_shared(&done_bar);

    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; ++s) {
            mbar_init(fb + 8 * s, 1);
            mbar_init(eb + 8 * s, 1);
        }
        mbar_init(db, 1);
        abort_s = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        const uint32_t slot = (uint32_t)__cvta_generic_to_shared(&tmem_slot);
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(slot),
                     "r"((uint32_t)BN)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_slot;

    if (threadIdx.x == 0) {
        // producer: TMA loads of stage s once the MMAs of its previous use are done
        for (int i = 0; i < nk; ++i) {
            const int s = i % kStages;
            const uint32_t ph = (uint32_t)(i / kStages) & 1u;
            if (i >= kStages && !mbar_wait(eb + 8 * s, ph ^ 1u)) {
                abort_s = 1;
                atomicExch(g.error_flag, 1);
                break;
            }
            if (*(volatile int*)&abort_s) break;
            mbar_expect_tx(fb + 8 * s, kABytes + kBBytes);
            const int kx = (kb0 + i) * kBK;
            tma_load_2d(sA + s * kABytes, &tmA, kx, m0, fb + 8 * s);
            tma_load_2d(sB + s * kBBytes, &tmB, kx, n0, fb + 8 * s);
        }
    } else if (threadIdx.x == 32) {
        // MMA issuer: four K = 16 steps per stage, then hand the stage back
        constexpr uint32_t idesc = bf16_idesc(kBM, BN);
        for (int i = 0; i < nk; ++i) {
            const int s = i % kStages;
            const uint32_t ph = (uint32_t)(i / kStages) & 1u;
            if (!mbar_wait(fb + 8 * s, ph) || *(volatile int*)&abort_s) {
                abort_s = 1;
                atomicExch(g.error_flag, 1);
                break;
            }
            tc_fence_after();
#pragma unroll
            for (int kk = 0; kk < kBK / 16; ++kk)
                umma_bf16(tmem, sw128_desc(sA + s * kABytes + kk * 32),
                          sw128_desc(sB + s * kBBytes + kk * 32), idesc,
                          (i > 0 || kk > 0) ? 1u : 0u);
            umma_commit(eb + 8 * s);
        }
        // arrives once every MMA issued above has completed
        umma_commit(db);
    }
    __syncwarp();

    // epilogue: warp w reads accumulator rows 32w..32w+31
    bool ok = mbar_wait(db, 0u);
    ok = __all_sync(0xffffffffu, ok) && !*(volatile int*)&abort_s;
    if (!ok && lane == 0) atomicExch(g.error_flag, 1);
    tc_fence_after();
    if (ok) {
        const int m = m0 + warp * 32 + lane;
        const bool add = g.out_mode == PN_OUT_F32_ADD;
        const bool use_bias = g.bias != nullptr && (!add || blockIdx.z == 0);
        const bool bf16_out = g.out_mode == PN_OUT_BF16;
        // row-major stores of 16 whole columns go out as 16-byte vectors when the
        // row's first element is 16-byte aligned
        const bool vec = !add && !g.transpose_out &&
                         ((reinterpret_cast<uintptr_t>(g.out) & 15u) == 0u) &&
                         (g.ldo % (bf16_out ? 8 : 4)) == 0;
#pragma unroll 1
        for (int c = 0; c < BN; c += 16) {
            float v[16];
            tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c, v);
            if (m >= g.M) continue;
            if (vec && n0 + c + 16 <= g.N) {
                const long long o = (long long)m * g.ldo + n0 + c;
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    float x = v[j];
                    if (use_bias) x += g.bias[n0 + c + j];
                    if (g.relu) x = fmaxf(x, 0.0f);
                    if (g.mask != nullptr && !(__bfloat162float(g.mask[o + j]) > 0.0f)) x = 0.0f;
                    v[j] = x;
                }
                if (bf16_out) {
                    uint32_t w[8];
#pragma unroll
                    for (int j = 0; j < 8; ++j) {
                        const __nv_bfloat162 h = __floats2bfloat162_rn(v[2 * j], v[2 * j + 1]);
                        w[j] = *reinterpret_cast<const uint32_t*>(&h);
                    }
                    uint4* dst = reinterpret_cast<uint4*>(reinterpret_cast<__nv_bfloat16*>(g.out) + o);
                    dst[0] = make_uint4(w[0], w[1], w[2], w[3]);
                    dst[1] = make_uint4(w[4], w[5], w[6], w[7]);
                } else {
                    float4* dst = reinterpret_cast<float4*>(reinterpret_cast<float*>(g.out) + o);
#pragma unroll
                    for (int j = 0; j < 4; ++j)
                        dst[j] = make_float4(v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]);
                }
                continue;
            }
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                const int n = n0 + c + j;
                if (n >= g.N) continue;
                float x = v[j];
                if (use_bias) x += g.bias[n];
                if (g.relu) x = fmaxf(x, 0.0f);
                if (g.mask != nullptr &&
                    !(__bfloat162float(g.mask[(long long)m * g.ldo + n]) > 0.0f))
                    x = 0.0f;
                const long long o = g.transpose_out ? (long long)n * g.ldo + m
                                                    : (long long)m * g.ldo + n;
                if (g.out_mode == PN_OUT_BF16)
                    reinterpret_cast<__nv_bfloat16*>(g.out)[o] = __float2bfloat16(x);
                else if (add)
                    atomicAdd(reinterpret_cast<float*>(g.out) + o, x);
                else
                    reinterpret_cast<float*>(g.out)[o] = x;
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                     "r"((uint32_t)BN)
                     : "memory");
}

// ---- host side of the GEMM ----------------------------------------------------

PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;
std::once_flag g_encode_once;
cudaError_t g_encode_err = cudaSuccess;

cudaError_t load_encode() {
    std::call_once(g_encode_once, [] {
        cudaDriverEntryPointQueryResult q;
        void* fn = nullptr;
        g_encode_err = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q);
        if (g_encode_err == cudaSuccess && (q != cudaDriverEntryPointSuccess || !fn))
            g_encode_err = cudaErrorSymbolNotFound;
        g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    });
    return g_encode_err;
}

// A rows x cols bf16 matrix with row stride ld (elements), read in boxes of
// box_rows x 64: rows past the end and columns past `cols` read as zero.
int make_tmap(CUtensorMap* tm, const void* ptr, long long rows, long long cols, long long ld,
              int box_rows) {
    if (!ptr || rows < 1 || cols < 1 || ld < cols || (ld * 2) % 16 != 0 ||
        (reinterpret_cast<uintptr_t>(ptr) & 15u) != 0)
        return PN_E_INVALID;
    cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)(ld * 2)};
    cuuint32_t box[2] = {(cuuint32_t)kBK, (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = g_encode(tm, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(ptr), dims,
                          strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                          CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? PN_OK : PN_E_INVALID;
}

template <int BN>
size_t gemm_smem() {
    return (size_t)kStages * (kBM * kBK * 2 + BN * kBK * 2) + 1024;
}

template <int BN>
int launch_gemm_bn(const CUtensorMap& ta, const void* B, long long ldb, const GemmArgs& g,
                   int splits, cudaStream_t st) {
    CUtensorMap tb;
    int rc = make_tmap(&tb, B, g.N, g.K, ldb, BN);
    if (rc) return rc;
    static std::once_flag once;
    static cudaError_t attr_err = cudaSuccess;
    std::call_once(once, [] {
        attr_err = cudaFuncSetAttribute(pn_gemm_kernel<BN>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)gemm_smem<BN>());
    });
    if (attr_err != cudaSuccess) return PN_E_CUDA;
    dim3 grid((g.M + kBM - 1) / kBM, (g.N + BN - 1) / BN, splits);
    pn_gemm_kernel<BN><<<grid, kGemmThreads, gemm_smem<BN>(), st>>>(ta, tb, g);
    return cudaGetLastError() == cudaSuccess ? PN_OK : PN_E_CUDA;
}

// ---- data movers and small steps ----------------------------------------------

// One CTA per curve: the curve binned into n_bins equal time bins over its own
// span.  Channel 0: the bin's mean flux minus the curve's mean, over the
// curve's standard deviation (0 for an empty bin); channel 1: 1 for an occupied
// bin.  out: [curve][bin][2] bf16.
__global__ void __launch_bounds__(256) bin_curves_kernel(const double* t, const double* y,
                                                         const long long* offsets, int n_bins,
                                                         __nv_bfloat16* out) {
    extern __shared__ float sbin[];     // 2 * n_bins: sum, count
    __shared__ double red[4][8];
    const int c = blockIdx.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const long long b = offsets[c], e = offsets[c + 1];
    const int n = (int)(e - b);
    double lo = INFINITY, hi = -INFINITY, s1 = 0.0, s2 = 0.0;
    for (int j = tid; j < n; j += blockDim.x) {
        const double tj = t[b + j], yj = y[b + j];
        lo = fmin(lo, tj);
        hi = fmax(hi, tj);
        s1 += yj;
        s2 += yj * yj;
    }
    for (int o = 16; o > 0; o >>= 1) {
        lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
        hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
        s1 += __shfl_xor_sync(0xffffffffu, s1, o);
        s2 += __shfl_xor_sync(0xffffffffu, s2, o);
    }
    if (lane == 0) {
        red[0][warp] = lo;
        red[1][warp] = hi;
        red[2][warp] = s1;
        red[3][warp] = s2;
    }
    for (int i = tid; i < 2 * n_bins; i += blockDim.x) sbin[i] = 0.0f;
    __syncthreads();
    lo = red[0][0];
    hi = red[1][0];
    s1 = 0.0;
    s2 = 0.0;
    for (int w = 0; w < 8; ++w) {
        lo = fmin(lo, red[0][w]);
        hi = fmax(hi, red[1][w]);
        s1 += red[2][w];
        s2 += red[3][w];
    }
    const double mean = n > 0 ? s1 / n : 0.0;
    const double var = n > 0 ? fmax(s2 / n - mean * mean, 0.0) : 0.0;
    const double inv_sd = var > 0.0 ? 1.0 / sqrt(var) : 0.0;
    const double span = hi - lo;
    const double scale = span > 0.0 ? (double)n_bins / span : 0.0;
    for (int j = tid; j < n; j += blockDim.x) {
        int k = (int)((t[b + j] - lo) * scale);
        k = k < 0 ? 0 : (k >= n_bins ? n_bins - 1 : k);
        atomicAdd(&sbin[2 * k], (float)((y[b + j] - mean) * inv_sd));
        atomicAdd(&sbin[2 * k + 1], 1.0f);
    }
    __syncthreads();
    __nv_bfloat16* o = out + (long long)c * n_bins * 2;
    for (int k = tid; k < n_bins; k += blockDim.x) {
        const float cnt = sbin[2 * k + 1];
        o[2 * k] = __float2bfloat16(cnt > 0.0f ? sbin[2 * k] / cnt : 0.0f);
        o[2 * k + 1] = __float2bfloat16(cnt > 0.0f ? 1.0f : 0.0f);
    }
}

// Rows (b, o) of the stride-2, width-7, padding-3 convolution's patches:
// A[(b * L_out + o), k * C + c] = X[b, 2o + k - 3, c] (0 outside), columns past
// 7C up to kp zero.  Each thread writes 8 consecutive bf16.
__global__ void im2col_kernel(const __nv_bfloat16* X, __nv_bfloat16* A, int B, int L_in, int C,
                              int kp) {
    const int L_out = L_in / 2;
    const long long chunks = (long long)kp / 8;
    const long long total = (long long)B * L_out * chunks;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const long long r = idx / chunks;
        const int col0 = (int)(idx - r * chunks) * 8;
        const int b = (int)(r / L_out), o = (int)(r - (long long)b * L_out);
        __align__(16) __nv_bfloat16 v[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) {
            const int col = col0 + e;
            __nv_bfloat16 x = __float2bfloat16(0.0f);
            if (col < 7 * C) {
                const int k = col / C, ch = col - k * C;
                const int i = 2 * o + k - 3;
                if (i >= 0 && i < L_in) x = X[((long long)b * L_in + i) * C + ch];
            }
            v[e] = x;
        }
        *reinterpret_cast<uint4*>(A + r * kp + col0) = *reinterpret_cast<const uint4*>(v);
    }
}

// The input gradient of that convolution: dX[b, i, c] = sum over taps k with
// i + 3 - k = 2o, 0 <= o < L_out, of dcol[(b * L_out + o), k * C + c], times
// (act[b, i, c] > 0) when act is given (the ReLU that produced X).
__global__ void col2im_kernel(const __nv_bfloat16* dcol, const __nv_bfloat16* act,
                              __nv_bfloat16* dX, int B, int L_in, int C, int kp) {
    const int L_out = L_in / 2;
    const long long total = (long long)B * L_in * C;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const int ch = (int)(idx % C);
        const long long bi = idx / C;
        const int i = (int)(bi % L_in);
        const int b = (int)(bi / L_in);
        float s = 0.0f;
#pragma unroll
        for (int k = 0; k < 7; ++k) {
            const int u = i + 3 - k;
            if (u < 0 || (u & 1)) continue;
            const int o = u >> 1;
            if (o >= L_out) continue;
            s += __bfloat162float(dcol[((long long)b * L_out + o) * kp + k * C + ch]);
        }
        if (act != nullptr && !(__bfloat162float(act[idx]) > 0.0f)) s = 0.0f;
        dX[idx] = __float2bfloat16(s);
    }
}

// out[c, r] = in[r, c] for r < R, c < C (bf16), 32 x 32 tiles through shared memory.
__global__ void transpose_kernel(const __nv_bfloat16* in, long long ld_in, __nv_bfloat16* out,
                                 long long ld_out, long long R, long long C) {
    __shared__ __nv_bfloat16 tile[32][33];
    const long long r0 = (long long)blockIdx.y * 32, c0 = (long long)blockIdx.x * 32;
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const long long r = r0 + k, c = c0 + threadIdx.x;
        tile[k][threadIdx.x] = (r < R && c < C) ? in[r * ld_in + c] : __float2bfloat16(0.0f);
    }
    __syncthreads();
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const long long c = c0 + k, r = r0 + threadIdx.x;
        if (c < C && r < R) out[c * ld_out + r] = tile[threadIdx.x][k];
    }
}

// db[n] += sum over rows of g[m, n] (bf16 g, ld), fp32 atomics per block.
__global__ void colsum_kernel(const __nv_bfloat16* g, long long ld, long long M, int N,
                              float* db) {
    const int n = blockIdx.y * blockDim.x + threadIdx.x;
    if (n >= N) return;
    const long long rows_per = (M + gridDim.x - 1) / gridDim.x;
    const long long a = blockIdx.x * rows_per, e = min(M, a + rows_per);
    float s = 0.0f;
    for (long long m = a; m < e; ++m) s += __bfloat162float(g[m * ld + n]);
    atomicAdd(db + n, s);
}

// One CTA per row of logits: the loss against a target spread over the label's
// bin (1 - 2 * side) and its two neighbours (side each, folded back at the
// ends), and dlogits = (softmax - target) * scale as bf16.
__global__ void __launch_bounds__(256) softmax_xent_kernel(const float* logits, int n_cls,
                                                           const int* labels, float side,
                                                           float scale, __nv_bfloat16* dlogits,
                                                           float* loss) {
    __shared__ float red[8];
    const int r = blockIdx.x, tid = threadIdx.x;
    const float* x = logits + (long long)r * n_cls;
    float mx = -INFINITY;
    for (int i = tid; i < n_cls; i += blockDim.x) mx = fmaxf(mx, x[i]);
    for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if ((tid & 31) == 0) red[tid >> 5] = mx;
    __syncthreads();
    mx = red[0];
    for (int w = 1; w < 8; ++w) mx = fmaxf(mx, red[w]);
    __syncthreads();
    float se = 0.0f;
    for (int i = tid; i < n_cls; i += blockDim.x) se += expf(x[i] - mx);
    for (int o = 16; o > 0; o >>= 1) se += __shfl_xor_sync(0xffffffffu, se, o);
    if ((tid & 31) == 0) red[tid >> 5] = se;
    __syncthreads();
    se = 0.0f;
    for (int w = 0; w < 8; ++w) se += red[w];
    const float lse = mx + logf(se);
    const int lab = labels[r];
    auto target = [&](int i) -> float {
        float p = 0.0f;
        if (i == lab) p += 1.0f - 2.0f * side;
        if (i == lab - 1 || (lab == 0 && i == 0)) p += side;
        if (i == lab + 1 || (lab == n_cls - 1 && i == n_cls - 1)) p += side;
        return p;
    };
    float l = 0.0f;
    for (int i = tid; i < n_cls; i += blockDim.x) {
        const float tg = target(i);
        const float p = expf(x[i] - lse);
        dlogits[(long long)r * n_cls + i] = __float2bfloat16((p - tg) * scale);
        if (tg > 0.0f) l -= tg * (x[i] - lse);
    }
    for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
    __syncthreads();
    if ((tid & 31) == 0) red[tid >> 5] = l;
    __syncthreads();
    if (tid == 0) {
        float s = 0.0f;
        for (int w = 0; w < 8; ++w) s += red[w];
        atomicAdd(loss, s);
    }
}

// Adam with decoupled weight decay on fp32 master weights; the bf16 copy the
// GEMMs read is refreshed in the same pass.
__global__ void adam_kernel(float* w, float* m, float* v, const float* g, __nv_bfloat16* w16,
                            long long n, float lr, float b1, float b2, float eps, float wd,
                            float c1, float c2) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.0f - b1) * gi;
        const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float wi = w[i] - lr * ((mi / c1) / (sqrtf(vi / c2) + eps) + wd * w[i]);
        w[i] = wi;
        if (w16 != nullptr) w16[i] = __float2bfloat16(wi);
    }
}

// One CTA per curve: the k largest logits (largest first; ties to the lower
// index) and the softmax probability mass they hold.
__global__ void __launch_bounds__(256) topk_kernel(const float* logits, int n_cls, int k,
                                                   int* index, float* mass) {
    extern __shared__ float sx[];
    __shared__ float rv[8];
    __shared__ int ri[8];
    const int r = blockIdx.x, tid = threadIdx.x;
    const float* x = logits + (long long)r * n_cls;
    float mx = -INFINITY;
    for (int i = tid; i < n_cls; i += blockDim.x) {
        sx[i] = x[i];
        mx = fmaxf(mx, x[i]);
    }
    for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if ((tid & 31) == 0) rv[tid >> 5] = mx;
    __syncthreads();
    mx = rv[0];
    for (int w = 1; w < 8; ++w) mx = fmaxf(mx, rv[w]);
    __syncthreads();
    float se = 0.0f;
    for (int i = tid; i < n_cls; i += blockDim.x) se += expf(sx[i] - mx);
    for (int o = 16; o > 0; o >>= 1) se += __shfl_xor_sync(0xffffffffu, se, o);
    __syncthreads();
    if ((tid & 31) == 0) rv[tid >> 5] = se;
    __syncthreads();
    se = 0.0f;
    for (int w = 0; w < 8; ++w) se += rv[w];
    float held = 0.0f;
    for (int q = 0; q < k; ++q) {
        float bv = -INFINITY;
        int bi = n_cls;
        for (int i = tid; i < n_cls; i += blockDim.x)
            if (sx[i] > bv || (sx[i] == bv && i < bi)) { bv = sx[i]; bi = i; }
        for (int o = 16; o > 0; o >>= 1) {
            const float ov = __shfl_xor_sync(0xffffffffu, bv, o);
            const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
            if (ov > bv || (ov == bv && oi < bi)) { bv = ov; bi = oi; }
        }
        __syncthreads();
        if ((tid & 31) == 0) { rv[tid >> 5] = bv; ri[tid >> 5] = bi; }
        __syncthreads();
        if (tid == 0) {
            for (int w = 1; w < 8; ++w)
                if (rv[w] > bv || (rv[w] == bv && ri[w] < bi)) { bv = rv[w]; bi = ri[w]; }
            index[(long long)r * k + q] = bi;
            if (bi < n_cls) {
                held += expf(bv - mx) / se;
                sx[bi] = -INFINITY;
            }
        }
        __syncthreads();
    }
    if (tid == 0) mass[r] = held;
}

int grid_for(long long n, int threads) {
    long long b = (n + threads - 1) / threads;
    return (int)(b < 1 ? 1 : (b > 148 * 32 ? 148 * 32 : b));
}

}  // namespace
}  // namespace pn
}  // namespace blsb200

using namespace blsb200::pn;

extern "C" {

int pn_gemm(const void* A, long long lda, const void* B, long long ldb, int M, int N, int K,
            int splits, void* out, long long ldo, int out_mode, int transpose_out,
            const float* bias, int relu, const void* mask, int* error_flag, void* stream) {
    if (M < 1 || N < 1 || K < 1 || !out || !error_flag || splits < 1) return PN_E_INVALID;
    if (out_mode == PN_OUT_F32_ADD && relu) return PN_E_INVALID;
    if (out_mode == PN_OUT_F32_ADD && mask) return PN_E_INVALID;
    if (load_encode() != cudaSuccess || !g_encode) return PN_E_CUDA;
    CUtensorMap ta;
    int rc = make_tmap(&ta, A, M, K, lda, kBM);
    if (rc) return rc;
    const int nk = (K + kBK - 1) / kBK;
    splits = splits > nk ? nk : splits;
    if (out_mode != PN_OUT_F32_ADD) splits = 1;
    GemmArgs g;
    g.M = M;
    g.N = N;
    g.K = K;
    g.kb_per_split = (nk + splits - 1) / splits;
    splits = (nk + g.kb_per_split - 1) / g.kb_per_split;
    g.out = out;
    g.ldo = ldo;
    g.out_mode = out_mode;
    g.transpose_out = transpose_out;
    g.bias = bias;
    g.relu = relu;
    g.mask = reinterpret_cast<const __nv_bfloat16*>(mask);
    g.error_flag = error_flag;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    if (N <= 64) return launch_gemm_bn<64>(ta, B, ldb, g, splits, st);
    if (N <= 128) return launch_gemm_bn<128>(ta, B, ldb, g, splits, st);
    return launch_gemm_bn<256>(ta, B, ldb, g, splits, st);
}

int pn_bin_curves(const double* t, const double* y, const long long* offsets, int n_curves,
                  int n_bins, void* out, void* stream) {
    if (n_curves < 1 || n_bins < 1 || n_bins > 8192 || !t || !y || !offsets || !out)
        return PN_E_INVALID;
    const size_t smem = (size_t)2 * n_bins * sizeof(float);
    if (smem > 48 * 1024 &&
        cudaFuncSetAttribute(bin_curves_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem) != cudaSuccess)
        return PN_E_CUDA;
    bin_curves_kernel<<<n_curves, 256, smem, reinterpret_cast<cudaStream_t>(stream)>>>(
        t, y, reinterpret_cast<const long long*>(offsets), n_bins,
        reinterpret_cast<__nv_bfloat16*>(out));
    return cudaGetLastError() == cudaSuccess ? PN_OK : PN_E_CUDA;
}

int pn_im2col(const void* X, void* A, int B, int L_in, int C, int kp, void* stream) {
    if (B < 1 || L_in < 2 || (L_in & 1) || C < 1 || kp < 7 * C || (kp % 8) != 0 || !X || !A)
        return PN_E_INVALID;
    const long long total = (long long)B * (L_in / 2) * (kp / 8);
    im2col_kernel<<<grid_for(total, 256), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        reinterpret_cast<const __nv_bfloat16*>(X), reinterpret_cast<__nv_bfloat16*>(A), B, L_in,
        C, kp);
    return cudaGetLastError() == cudaSuccess ? PN_OK : PN_E_CUDA;
}

int pn_col2im(const void* dcol, const void* act, void* dX, int B, int L_in, int C, int kp,
              void* stream) {
    if (B < 1 || L_in < 2 || (L_in & 1) || C < 1 || kp < 7 * C || !dcol || !dX)
        return PN_E_INVALID;
    const long long total = (long long)B * L_in * C;
    col2im_kernel<<<grid_for(total, 256), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        reinterpret_cast<const __nv_bfloat16*>(dcol), reinterpret_cast<const __nv_bfloat16*>(act),
        reinterpret_cast<__nv_bfloat16*>(dX), B, L_in, C, kp);
    return cudaGetLastError() == cudaSuccess ? PN_OK : PN_E_CUDA;
}

int pn_transpose(const void* in, long long ld_in, void* out, long long ld_out, long long R,
                 long long C, void* stream) {
    if (R < 1 || C < 1 || !in || !out || ld_in < C || ld_out < R) return PN_E_INVALID;
    if ((C + 31) / 32 > 0x7fffffffll || (R + 31) / 32 > 65535) return PN_E_INVALID;
    dim3 grid((unsigned)((C + 31) / 32), (unsigned)((R + 31) / 32));
    transpose_kernel<<<grid, dim3(32, 8), 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        reinterpret_cast<const __nv_bfloat16*>(in), ld_in, reinterpret_cast<__nv_bfloat16*>(out),
        ld_out, R, C);
    return cudaGetLastError() == cudaSuccess ? PN_OK : PN_E_CUDA;
}

int pn_colsum(const void* g, long long ld, long long M, int N, float* db, void* stream) {
    if (M < 1 || N < 1 || !g || !db || ld < N) return PN_E_INVALID;
    dim3 grid((unsigned)(M < 1024 ? 1 : (M / 1024 > 4096 ? 4096 : M / 1024)),
              (unsigned)((N + 127) / 128));
    colsum_kernel<<<grid, 128, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        reinterpret_cast<const __nv_bfloat16*>(g), ld, M, N, db);
    return cudaGetLastError() == cudaSuccess ? PN_OK : PN_E_CUDA;
}

int pn_softmax_xent(const float* logits, int rows, int n_cls, const int* labels, float side,
                    float scale, void* dlogits, float* loss, void* stream) {
    if (rows < 1 || n_cls < 3 || !logits || !labels || !dlogits || !loss || side < 0.0f ||
        side > 0.5f)
        return PN_E_INVALID;
    softmax_xent_kernel<<<rows, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        logits, n_cls, labels, side, scale, reinterpret_cast<__nv_bfloat16*>(dlogits), loss);
    return cudaGetLastError() == cudaSuccess ? PN_OK : PN_E_CUDA;
}

int pn_adam(float* w, float* m, float* v, const float* g, void* w16, long long n, float lr,
            float b1, float b2, float eps, float wd, int step, void* stream) {
    if (n < 1 || !w || !m || !v || !g || step < 1) return PN_E_INVALID;
    const float c1 = 1.0f - powf(b1, (float)step), c2 = 1.0f - powf(b2, (float)step);
    adam_kernel<<<grid_for(n, 256), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        w, m, v, g, reinterpret_cast<__nv_bfloat16*>(w16), n, lr, b1, b2, eps, wd, c1, c2);
    return cudaGetLastError() == cudaSuccess ? PN_OK : PN_E_CUDA;
}

int pn_topk(const float* logits, int rows, int n_cls, int k, int* index, float* mass,
            void* stream) {
    if (rows < 1 || n_cls < 1 || n_cls > 16384 || k < 1 || k > n_cls || !logits || !index ||
        !mass)
        return PN_E_INVALID;
    topk_kernel<<<rows, 256, (size_t)n_cls * sizeof(float),
                  reinterpret_cast<cudaStream_t>(stream)>>>(logits, n_cls, k, index, mass);
    return cudaGetLastError() == cudaSuccess ? PN_OK : PN_E_CUDA;
}

}  // extern "C"
