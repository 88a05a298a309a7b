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
#include <math.h>
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

// Fold probe: the search kernel's fast fold path alone, on one synthetic
// one-weight curve (10,240 points at a 2-minute cadence with 5% dropouts) and
// eight periods of 0.3-0.6 d with 0.001 d bins (611-bin histograms, 12-byte
// records, the kernel's layout), each CTA folding it kFoldItems times.
// Variant 0: the phase, the edge tests and the record address only; 1: plus
// three atomics per point; 2: plus the merging of runs of equal bins before
// the atomics, as the kernel does.  Every record address stays inside its
// period's histogram: S <= 600.1 * 2^22, so (S - 1) >> 22 + 1 <= 601 < 611.
constexpr int kFoldThreads = 256, kFoldPts = 8, kFoldPeriods = 8, kFoldBins = 611;
constexpr int kFoldItems = 64, kFoldN = 10240;
constexpr int kFoldRec = 12;
constexpr uint32_t kFoldPeriodBytes = ((kFoldBins * kFoldRec + 15) / 16) * 16;

template <int OFF>
__device__ __forceinline__ void probe_red(uint32_t a, uint32_t v) {
    asm volatile("red.shared.add.u32 [%0+%2], %1;" ::"r"(a), "r"(v), "n"(OFF) : "memory");
}

template <int V>
__global__ void __launch_bounds__(kFoldThreads, 3)
    fold_probe(const double* __restrict__ tau, const uint32_t* __restrict__ pay,
               const double* __restrict__ fq, const uint32_t* __restrict__ sq,
               uint32_t* sink) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ double s_f[kFoldPeriods];
    __shared__ uint32_t s_S[kFoldPeriods];
    const int tid = threadIdx.x;
    if (tid < kFoldPeriods) {
        s_f[tid] = fq[tid];
        s_S[tid] = sq[tid];
    }
    const uint32_t hist_s = (uint32_t)__cvta_generic_to_shared(smem);
    const int fb = 22;
    const uint32_t fmask = (1u << fb) - 1u, mu = 5u, fr_span = (1u << fb) - 10u;
    const uint32_t mphi = 3u, phi_span = 0u - 6u;
    constexpr uint32_t kB = kFoldRec;
    uint32_t acc = 0;
    for (int it = 0; it < kFoldItems; ++it) {
        for (int i = tid; i < (int)(kFoldPeriods * kFoldPeriodBytes / 16); i += kFoldThreads)
            reinterpret_cast<uint4*>(smem)[i] = make_uint4(0u, 0u, 0u, 0u);
        __syncthreads();
        for (int base = 0; base < kFoldN; base += kFoldThreads * kFoldPts) {
            double x[kFoldPts];
            uint32_t lo[kFoldPts], hi[kFoldPts];
#pragma unroll
            for (int r = 0; r < kFoldPts; ++r) {
                const int j = base + r * kFoldThreads + tid;
                x[r] = __ldg(tau + j);
                const uint32_t w = __ldg(pay + j);
                lo[r] = w & 0xffffu;
                hi[r] = (uint32_t)((int32_t)w >> 16);
            }
            for (int q = 0; q < kFoldPeriods; ++q) {
                const double f = s_f[q];
                const uint32_t S = s_S[q];
                const uint32_t hq = hist_s + (uint32_t)q * kFoldPeriodBytes;
                uint32_t rec[kFoldPts];
                bool all_ok = true;
#pragma unroll
                for (int r = 0; r < kFoldPts; ++r) {
                    const double qm = __fma_rn(x[r], f, 1572864.0);
                    const uint32_t phi = (uint32_t)__double2loint(qm);
                    const uint32_t v = __umulhi(phi, S);
                    all_ok &= ((phi - mphi) < phi_span) & (((v & fmask) - mu) < fr_span);
                    rec[r] = hq + kB + (v >> fb) * kB;
                }
                if (V == 0) {
#pragma unroll
                    for (int r = 0; r < kFoldPts; ++r) acc += all_ok ? rec[r] : 1u;
                } else if (!all_ok) {
                    continue;
                } else if (V == 1) {
#pragma unroll
                    for (int r = 0; r < kFoldPts; ++r) {
                        probe_red<0>(rec[r], lo[r]);
                        probe_red<4>(rec[r], hi[r]);
                        probe_red<8>(rec[r], 1u);
                    }
                } else {
                    uint32_t s_lo = lo[0], s_hi = hi[0], s_c = 1u;
#pragma unroll
                    for (int r = 1; r < kFoldPts; ++r) {
                        if (rec[r] != rec[r - 1]) {
                            probe_red<0>(rec[r - 1], s_lo);
                            probe_red<4>(rec[r - 1], s_hi);
                            probe_red<8>(rec[r - 1], s_c);
                            s_lo = 0u;
                            s_hi = 0u;
                            s_c = 0u;
                        }
                        s_lo += lo[r];
                        s_hi += hi[r];
                        s_c += 1u;
                    }
                    probe_red<0>(rec[kFoldPts - 1], s_lo);
                    probe_red<4>(rec[kFoldPts - 1], s_hi);
                    probe_red<8>(rec[kFoldPts - 1], s_c);
                }
            }
        }
        __syncthreads();
        acc += reinterpret_cast<const uint32_t*>(smem)[tid];
        __syncthreads();
    }
    sink[blockIdx.x * kFoldThreads + tid] = acc;
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


// Runs the fold probe's three variants (three CTAs per SM), each once to warm up
// and once timed with CUDA events, and writes one line per variant: name,
// milliseconds, point-folds per second (1e9).  Returns 0 or a CUDA error code.
int bls_probe_fold(char* report, int report_len) {
    int dev = 0, n_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
    const int blocks = 3 * n_sm;
    // the curve: a 2-minute cadence with a seeded 5% of dropouts, and one-weight
    // payload words (13-bit low part, small signed high part)
    double* h_tau = new double[kFoldN];
    uint32_t* h_pay = new uint32_t[kFoldN];
    uint32_t rnd = 12345u;
    int n = 0;
    for (int k = 0; n < kFoldN; ++k) {
        rnd = rnd * 1664525u + 1013904223u;
        if ((rnd >> 8) % 100u < 5u) continue;
        h_tau[n] = k * (2.0 / 1440.0);
        rnd = rnd * 1664525u + 1013904223u;
        const uint32_t lo = (rnd >> 9) & 8191u;
        const int32_t hi = (int32_t)((rnd >> 3) % 601u) - 300;
        h_pay[n] = lo | ((uint32_t)(uint16_t)(int16_t)hi << 16);
        ++n;
    }
    double h_f[kFoldPeriods];
    uint32_t h_S[kFoldPeriods];
    for (int q = 0; q < kFoldPeriods; ++q) {
        const double P = 0.3 * pow(2.0, q / 7.0);          // 0.3 .. 0.6 d
        h_f[q] = 1.0 / P;
        h_S[q] = (uint32_t)llrint(P / 0.001 * 4194304.0);
    }
    double *tau = nullptr, *fq = nullptr;
    uint32_t *pay = nullptr, *sq = nullptr, *sink = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaError_t e = cudaMalloc(&tau, sizeof(double) * kFoldN);
    if (e == cudaSuccess) e = cudaMalloc(&pay, sizeof(uint32_t) * kFoldN);
    if (e == cudaSuccess) e = cudaMalloc(&fq, sizeof(h_f));
    if (e == cudaSuccess) e = cudaMalloc(&sq, sizeof(h_S));
    if (e == cudaSuccess) e = cudaMalloc(&sink, sizeof(uint32_t) * blocks * kFoldThreads);
    if (e == cudaSuccess) e = cudaMemcpy(tau, h_tau, sizeof(double) * kFoldN, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(pay, h_pay, sizeof(uint32_t) * kFoldN, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(fq, h_f, sizeof(h_f), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(sq, h_S, sizeof(h_S), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    const size_t smem = (size_t)kFoldPeriods * kFoldPeriodBytes;
    const double folds = (double)blocks * kFoldItems * kFoldN * kFoldPeriods;
    int pos = 0;
    auto run = [&](const char* name, auto kernel) {
        if (e != cudaSuccess) return;
        e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return;
        kernel<<<blocks, kFoldThreads, smem>>>(tau, pay, fq, sq, sink);
        cudaEventRecord(e0);
        kernel<<<blocks, kFoldThreads, smem>>>(tau, pay, fq, sq, sink);
        cudaEventRecord(e1);
        e = cudaEventSynchronize(e1);
        if (e == cudaSuccess) e = cudaGetLastError();
        float ms = 0.0f;
        if (e == cudaSuccess) cudaEventElapsedTime(&ms, e0, e1);
        pos += snprintf(report + pos, report_len - pos, "%s %.3f %.1f\n", name, ms,
                        folds / (ms * 1e-3) / 1e9);
    };
    run("fold_phase_tests_address", fold_probe<0>);
    run("fold_plus_three_atomics", fold_probe<1>);
    run("fold_plus_run_merging", fold_probe<2>);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(tau);
    cudaFree(pay);
    cudaFree(fq);
    cudaFree(sq);
    cudaFree(sink);
    delete[] h_tau;
    delete[] h_pay;
    return (int)e;
}

}  // extern "C"
