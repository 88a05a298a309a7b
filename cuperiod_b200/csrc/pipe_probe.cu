// Pipe-rate probe for the BLS kernels' design: shared-memory atomic add
// throughput by type and address pattern, FP64 add/mul/divide, FP32 FMA,
// 32-bit multiply-high and the conversions the fold/scan/sweep use.
//
// Every probe kernel touches only its own shared array (indices masked to its
// size) and one global output slot per thread; every loop has a fixed trip
// count.  Results are per-SM rates in operations per SM clock, the clock taken
// from clock64() against %globaltimer inside the same kernel.
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

namespace {

constexpr int kHist = 2048;          // shared entries per block
constexpr int kIters = 4096;         // operations per thread per probe

__device__ __forceinline__ uint64_t globaltimer_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

struct Stamp { unsigned long long c0, c1, t0, t1; };

template <typename T, int kPattern>
__global__ void atomics_probe(T* sink, Stamp* st) {
    __shared__ T h[kHist];
    for (int i = threadIdx.x; i < kHist; i += blockDim.x) h[i] = T(0);
    __syncthreads();
    const unsigned long long c0 = clock64();
    const uint64_t t0 = globaltimer_ns();
    uint32_t a = 0x9E3779B9u * (threadIdx.x + 1) + blockIdx.x;
    const T one = T(1);
#pragma unroll 8
    for (int k = 0; k < kIters; ++k) {
        int idx;
        if (kPattern == 0) {               // pseudo-random bins
            a = a * 1664525u + 1013904223u;
            idx = (a >> 21) & (kHist - 1);
        } else if (kPattern == 1) {        // conflict-free: lane-consecutive bins
            idx = (threadIdx.x + k * 32) & (kHist - 1);
        } else {                           // neighbouring lanes ~1.4 bins apart
            idx = ((threadIdx.x * 7) / 5 + k * 45) & (kHist - 1);
        }
        atomicAdd(&h[idx], one);
    }
    __syncthreads();
    const unsigned long long c1 = clock64();
    const uint64_t t1 = globaltimer_ns();
    if (threadIdx.x == 0) {
        st[blockIdx.x] = Stamp{c0, c1, t0, t1};
    }
    T s = T(0);
    for (int i = threadIdx.x; i < kHist; i += blockDim.x) s += h[i];
    sink[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

// Arithmetic probes: 8 independent chains per thread.
template <int kOp>
__global__ void arith_probe(double* sink, Stamp* st, double seed) {
    double x[8];
    float f[8];
    uint32_t u[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        x[i] = seed + 0.001 * (threadIdx.x + i);
        f[i] = (float)x[i];
        u[i] = 0x12345u * (threadIdx.x + 7 * i + 1);
    }
    const double m = 1.0000001, c = 1e-9;
    __syncthreads();
    const unsigned long long c0 = clock64();
    const uint64_t t0 = globaltimer_ns();
    for (int k = 0; k < kIters / 8; ++k) {
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            if (kOp == 0) x[i] = __dadd_rn(x[i], c);              // DADD
            else if (kOp == 1) x[i] = __dmul_rn(x[i], m);         // DMUL
            else if (kOp == 2) x[i] = __fma_rn(x[i], m, c);       // DFMA
            else if (kOp == 3) x[i] = __ddiv_rn(x[i] + 3.0, x[i]); // IEEE divide
            else if (kOp == 4) f[i] = __fmaf_rn(f[i], 1.0000001f, 1e-7f);  // FFMA
            else if (kOp == 5) u[i] = __umulhi(u[i], 0x9E3779B9u) + u[i];  // IMAD.HI
            else if (kOp == 6) f[i] += __double2float_rn(x[i] + f[i]);     // F64->F32
            else if (kOp == 7) x[i] += __ll2double_rn((long long)u[i] + k);  // S64->F64
            else if (kOp == 8) x[i] = floor(x[i] * m);            // floor(F64)
        }
    }
    const unsigned long long c1 = clock64();
    const uint64_t t1 = globaltimer_ns();
    if (threadIdx.x == 0) st[blockIdx.x] = Stamp{c0, c1, t0, t1};
    double s = 0.0;
#pragma unroll
    for (int i = 0; i < 8; ++i) s += x[i] + f[i] + u[i];
    sink[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

}  // namespace

extern "C" {

// Runs every probe once on the current device and writes one line per probe:
// name, ops per SM clock (whole SM), SM MHz.  Returns 0 or a CUDA error code.
int bls_probe_pipes(char* report, int report_len) {
    int dev = 0, n_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
    const int threads = 512, blocks_per_sm = 2;
    const int n_blocks = n_sm * blocks_per_sm;
    double* sink = nullptr;
    Stamp* st = nullptr;
    cudaError_t e = cudaMalloc(&sink, sizeof(double) * n_blocks * threads);
    if (e != cudaSuccess) return (int)e;
    e = cudaMalloc(&st, sizeof(Stamp) * n_blocks);
    if (e != cudaSuccess) { cudaFree(sink); return (int)e; }
    Stamp* hst = new Stamp[n_blocks];
    int pos = 0;
    auto measure = [&](const char* name, double ops_per_thread, auto launch) {
        launch();  // warm-up
        launch();
        cudaError_t err = cudaDeviceSynchronize();
        if (err != cudaSuccess) return (int)err;
        cudaMemcpy(hst, st, sizeof(Stamp) * n_blocks, cudaMemcpyDeviceToHost);
        double cyc = 0.0, ns = 0.0;
        for (int b = 0; b < n_blocks; ++b) {
            cyc += (double)(hst[b].c1 - hst[b].c0);
            ns += (double)(hst[b].t1 - hst[b].t0);
        }
        cyc /= n_blocks;
        ns /= n_blocks;
        // blocks_per_sm blocks share one SM for the same interval
        const double per_sm_clk = ops_per_thread * threads * blocks_per_sm / cyc;
        pos += snprintf(report + pos, report_len - pos, "%s %.3f %.0f\n", name, per_sm_clk,
                        cyc / ns * 1e3);
        return 0;
    };
    int rc = 0;
#define ATOM(T, P, NAME) \
    if (!rc) rc = measure(NAME, kIters, [&] { \
        atomics_probe<T, P><<<n_blocks, threads>>>((T*)sink, st); });
    ATOM(unsigned int, 0, "smem_atomic_add_u32_random")
    ATOM(unsigned long long, 0, "smem_atomic_add_u64_random")
    ATOM(float, 0, "smem_atomic_add_f32_random")
    ATOM(double, 0, "smem_atomic_add_f64_random")
    ATOM(unsigned long long, 1, "smem_atomic_add_u64_consecutive")
    ATOM(double, 1, "smem_atomic_add_f64_consecutive")
    ATOM(unsigned long long, 2, "smem_atomic_add_u64_neighbour")
    ATOM(unsigned int, 1, "smem_atomic_add_u32_consecutive")
#undef ATOM
#define ARITH(OP, NAME) \
    if (!rc) rc = measure(NAME, kIters, [&] { \
        arith_probe<OP><<<n_blocks, threads>>>(sink, st, 1.5); });
    ARITH(0, "dadd")
    ARITH(1, "dmul")
    ARITH(2, "dfma")
    ARITH(3, "ddiv_rn")
    ARITH(4, "ffma")
    ARITH(5, "umulhi_u32")
    ARITH(6, "cvt_f64_to_f32")
    ARITH(7, "cvt_s64_to_f64")
    ARITH(8, "floor_f64")
#undef ARITH
    delete[] hst;
    cudaFree(sink);
    cudaFree(st);
    return rc;
}

}  // extern "C"
