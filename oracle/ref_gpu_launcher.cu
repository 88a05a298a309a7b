// TEST AND MEASUREMENT INFRASTRUCTURE ONLY -- not part of the engine.
//
// Host launcher of the reference's own GPU kernel, bls_block (cuPeriod
// src/cuperiod/methods/_bls_core.py:505-656), which build_ref_gpu.py extracts
// from the reference's source at build time and compiles for sm_100a into the
// same library, once per precision (bls_block_f64 and bls_block_f32, REAL and
// CUDA_BLOCK substituted as _cuda_kernel does, _bls_core.py:661-672).  The launcher does for one light
// curve what _bls_search_cuda_specs does (_bls_core.py:741-840): one upload of
// the curve and of every segment's periods and box widths, one launch per
// segment (one block of CUDA_BLOCK threads per trial period, 2 x width REALs of
// dynamic shared memory), one download of the (7, n_periods) FP64 output.
// Device buffers are kept between calls and grown on demand, as cupy's memory
// pool keeps them.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <vector>

// The kernel's argument list (_bls_core.py:506-517), once per precision.
#define REF_BLS_BLOCK_DECL(NAME, R)                                                          \
    extern "C" __global__ void NAME(                                                        \
        const R* __restrict__ tau, const R* __restrict__ yw, const R* __restrict__ wv,      \
        const R* __restrict__ periods, const int* __restrict__ dur_bins, const int n_points, \
        const int n_periods, const int n_dur, const R bin_duration, const int oversample,    \
        const int width, const R sum_y, const R sum_ivar, const double t_min,               \
        const int obj_flag, const R NEG_INF, const R IVAR_EPS, double* o_power,             \
        double* o_depth, double* o_depth_err, double* o_depth_snr, double* o_duration,      \
        double* o_transit_time, double* o_loglike);
REF_BLS_BLOCK_DECL(bls_block_f64, double)
REF_BLS_BLOCK_DECL(bls_block_f32, float)

namespace {

struct RefBuf {
    void* p = nullptr;
    size_t cap = 0;
    cudaError_t ensure(size_t bytes) {
        if (bytes <= cap) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
        cudaError_t e = cudaMalloc(&p, bytes);
        if (e == cudaSuccess) cap = bytes;
        return e;
    }
};

RefBuf g_tau, g_yw, g_iv, g_per, g_dur, g_out;
cudaStream_t g_stream = nullptr;
cudaEvent_t g_ev0 = nullptr, g_ev1 = nullptr;

template <typename REAL_T>
int run(const double* tau, const double* yw, const double* iv, int n, const double* periods,
        const int32_t* seg_sizes, const int32_t* dur_bins, const int32_t* dur_sizes,
        const double* bin_durs, const int32_t* widths, int n_seg, int oversample, int obj_flag,
        double sum_y, double sum_ivar, double t_min, double floor_v, double* out,
        float* kernel_ms) {
    cudaError_t e;
#define REF_TRY(x) do { e = (x); if (e != cudaSuccess) return (int)e; } while (0)
    if (!g_stream) {
        REF_TRY(cudaStreamCreateWithFlags(&g_stream, cudaStreamNonBlocking));
        REF_TRY(cudaEventCreate(&g_ev0));
        REF_TRY(cudaEventCreate(&g_ev1));
    }
    int64_t total = 0, dtotal = 0;
    for (int k = 0; k < n_seg; ++k) {
        total += seg_sizes[k];
        dtotal += dur_sizes[k];
    }
    std::vector<REAL_T> h_tau(n), h_yw(n), h_iv(n), h_per(total);
    for (int j = 0; j < n; ++j) {
        h_tau[j] = (REAL_T)tau[j];
        h_yw[j] = (REAL_T)yw[j];
        h_iv[j] = (REAL_T)iv[j];
    }
    for (int64_t p = 0; p < total; ++p) h_per[p] = (REAL_T)periods[p];
    const size_t rb = sizeof(REAL_T);
    REF_TRY(g_tau.ensure(rb * n + 16));
    REF_TRY(g_yw.ensure(rb * n + 16));
    REF_TRY(g_iv.ensure(rb * n + 16));
    REF_TRY(g_per.ensure(rb * total + 16));
    REF_TRY(g_dur.ensure(sizeof(int32_t) * dtotal + 16));
    REF_TRY(g_out.ensure(sizeof(double) * 7 * total + 16));
    cudaStream_t st = g_stream;
    REF_TRY(cudaMemcpyAsync(g_tau.p, h_tau.data(), rb * n, cudaMemcpyHostToDevice, st));
    REF_TRY(cudaMemcpyAsync(g_yw.p, h_yw.data(), rb * n, cudaMemcpyHostToDevice, st));
    REF_TRY(cudaMemcpyAsync(g_iv.p, h_iv.data(), rb * n, cudaMemcpyHostToDevice, st));
    REF_TRY(cudaMemcpyAsync(g_per.p, h_per.data(), rb * total, cudaMemcpyHostToDevice, st));
    REF_TRY(cudaMemcpyAsync(g_dur.p, dur_bins, sizeof(int32_t) * dtotal, cudaMemcpyHostToDevice,
                            st));
    auto kern = sizeof(REAL_T) == 8 ? (void*)bls_block_f64 : (void*)bls_block_f32;
    int dev = 0, optin = 0;
    REF_TRY(cudaGetDevice(&dev));
    REF_TRY(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    REF_TRY(cudaEventRecord(g_ev0, st));
    double* o = (double*)g_out.p;
    int64_t p_off = 0, d_off = 0;
    const REAL_T neg = (REAL_T)(-INFINITY);
    for (int k = 0; k < n_seg; ++k) {
        const int np_ = seg_sizes[k], nd = dur_sizes[k];
        if (np_ > 0 && nd > 0) {
            // core/backend.py:340-384: dynamic plus static shared memory within the
            // device's opt-in (else the reference refuses), the opt-in raised above 48 KB
            const size_t smem = 2 * (size_t)widths[k] * rb;
            cudaFuncAttributes fa;
            REF_TRY(cudaFuncGetAttributes(&fa, kern));
            const size_t needed = smem + fa.sharedSizeBytes;
            if (needed > (size_t)optin) return -1;
            if (needed > 48 * 1024)
                REF_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem));
            const REAL_T* a_tau = (const REAL_T*)g_tau.p;
            const REAL_T* a_yw = (const REAL_T*)g_yw.p;
            const REAL_T* a_iv = (const REAL_T*)g_iv.p;
            const REAL_T* a_per = (const REAL_T*)g_per.p + p_off;
            const int* a_dur = (const int*)g_dur.p + d_off;
            int n_points = n, n_periods = np_, n_dur = nd, ov = oversample, width = widths[k];
            int obj = obj_flag;
            REAL_T bin = (REAL_T)bin_durs[k], sy = (REAL_T)sum_y, si = (REAL_T)sum_ivar;
            REAL_T fl = (REAL_T)floor_v;
            double tm = t_min;
            double* outs[7];
            for (int f = 0; f < 7; ++f) outs[f] = o + (size_t)f * total + p_off;
            void* args[] = {&a_tau, &a_yw, &a_iv, &a_per, &a_dur, &n_points, &n_periods, &n_dur,
                            &bin, &ov, &width, &sy, &si, &tm, &obj, (void*)&neg, &fl,
                            &outs[0], &outs[1], &outs[2], &outs[3], &outs[4], &outs[5],
                            &outs[6]};
            REF_TRY(cudaLaunchKernel(kern, dim3(np_), dim3(REF_CUDA_BLOCK), args, smem, st));
        } else {
            // _empty_output: power -inf, zeros elsewhere
            std::vector<double> z((size_t)np_, 0.0), ni((size_t)np_, -INFINITY);
            for (int f = 0; f < 7; ++f)
                REF_TRY(cudaMemcpyAsync(o + (size_t)f * total + p_off, f == 0 ? ni.data() : z.data(),
                                        sizeof(double) * np_, cudaMemcpyHostToDevice, st));
            REF_TRY(cudaStreamSynchronize(st));
        }
        p_off += np_;
        d_off += nd;
    }
    REF_TRY(cudaEventRecord(g_ev1, st));
    REF_TRY(cudaMemcpyAsync(out, o, sizeof(double) * 7 * total, cudaMemcpyDeviceToHost, st));
    REF_TRY(cudaStreamSynchronize(st));
    REF_TRY(cudaGetLastError());
    if (kernel_ms) REF_TRY(cudaEventElapsedTime(kernel_ms, g_ev0, g_ev1));
#undef REF_TRY
    return 0;
}

}  // namespace

extern "C" {

// One light curve through the reference's GPU search: tau = t - t_min, yw = y*ivar
// and ivar (FP64 host arrays; cast to the kernel's REAL on the host as cupy's
// asarray(..., dtype=rdtype) does), the segments' periods concatenated, each
// segment's box widths in bins, bin duration and width.  precision 0 = the
// reference's default double kernel, 1 = its float32 opt-in.  out: 7 x n_periods
// FP64, field-major.  kernel_ms: device time from the first launch to the last
// kernel's end.  Returns 0, a CUDA error code, or -1 for a segment whose shared
// memory the device cannot give (the reference's BackendUnavailableError).
int ref_bls_search_curve(const double* tau, const double* yw, const double* iv, int n,
                         const double* periods, const int32_t* seg_sizes, const int32_t* dur_bins,
                         const int32_t* dur_sizes, const double* bin_durs, const int32_t* widths,
                         int n_seg, int oversample, int obj_flag, double sum_y, double sum_ivar,
                         double t_min, double floor_v, int precision, double* out,
                         float* kernel_ms) {
    if (precision == 1)
        return run<float>(tau, yw, iv, n, periods, seg_sizes, dur_bins, dur_sizes, bin_durs,
                          widths, n_seg, oversample, obj_flag, sum_y, sum_ivar, t_min, floor_v,
                          out, kernel_ms);
    return run<double>(tau, yw, iv, n, periods, seg_sizes, dur_bins, dur_sizes, bin_durs, widths,
                       n_seg, oversample, obj_flag, sum_y, sum_ivar, t_min, floor_v, out,
                       kernel_ms);
}

}  // extern "C"
