// TEST INFRASTRUCTURE ONLY -- an all-FP64 GPU restatement of cuPeriod's
// unscreened numba box search (src/cuperiod/methods/_bls_core.py:341-462,
// _bls_search_numba(..., screen=False)), bit for bit: the checker of the engine
// at sizes the CPU oracle cannot reach (the 4-year, 200,000-period workload).
// Only the tests and bench.py's precision checks load it; the engine never does.
//
// One warp per trial period, the histogram in shared memory:
//   fold   -- points 32 at a time in index order; lane l takes point 32i + l and
//             computes the reference's bin with its own IEEE operations
//             (w = x - P*floor(x/P); ind = int(w/bin) + 1, clipped, no
//             contraction: this file is built with -fmad=false); lanes that
//             share a bin are grouped (__match_any_sync) and the group's lowest
//             lane adds their values to the bin one after another in lane order,
//             so every bin is the reference's sequential sum in point order;
//   pad    -- bins 1..o copied to n_bins-o..n_bins-1 by lane 0, in order;
//   prefix -- the running sums by lane 0, in bin order;
//   sweep  -- every (duration, start) box by the lanes in parallel with the
//             reference's FP64 formulas; the winner is the largest objective,
//             ties to the earliest (duration index, start) -- the reference's
//             strict "obj > loc" in its loop order;
//   epilogue -- lane 0, the reference's seven fields.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

namespace {

__device__ __forceinline__ bool before(double v, int di, int n, double w, int dj, int m) {
    if (v > w) return true;
    if (!(v == w)) return false;
    return di < dj || (di == dj && n < m);
}

__global__ void __launch_bounds__(32) oracle_period_kernel(
    const double* __restrict__ tau, const double* __restrict__ yw, const double* __restrict__ wv,
    int n_points, const double* __restrict__ periods, int n_periods,
    const int64_t* __restrict__ dur_bins, int n_dur, double bin_duration, int oversample,
    int width, double sum_y, double sum_ivar, double t_min, int obj_flag, double ivar_floor,
    double* __restrict__ out) {
    extern __shared__ double sh[];
    double* my = sh;
    double* mi = sh + width;
    const int pidx = blockIdx.x;
    if (pidx >= n_periods) return;
    const int lane = threadIdx.x;
    const double period = periods[pidx];
    int n_bins = (int)ceil(period / bin_duration) + oversample;
    if (n_bins > width - 1) n_bins = width - 1;
    for (int i = lane; i <= n_bins; i += 32) {
        my[i] = 0.0;
        mi[i] = 0.0;
    }
    __syncwarp();
    for (int base = 0; base < n_points; base += 32) {
        const int j = base + lane;
        const bool ok = j < n_points;
        int ind = -1;
        double vy = 0.0, vi = 0.0;
        if (ok) {
            const double x = tau[j];
            const double w = x - period * floor(x / period);
            ind = (int)(w / bin_duration) + 1;
            if (ind < 0) ind = 0;
            else if (ind > width - 1) ind = width - 1;
            vy = yw[j];
            vi = wv[j];
        }
        const unsigned grp = __match_any_sync(0xffffffffu, ind);
        const int leader = __ffs(grp) - 1;
        // every lane of a group hands its values to the leader in lane order
        double ay = 0.0, ai = 0.0;
        if (ok && lane == leader) {
            ay = my[ind];
            ai = mi[ind];
        }
        for (unsigned m = grp; m != 0u; m &= m - 1u) {
            const int src = __ffs(m) - 1;
            const double sy = __shfl_sync(grp, vy, src);
            const double si = __shfl_sync(grp, vi, src);
            if (lane == leader) {
                ay += sy;
                ai += si;
            }
        }
        if (ok && lane == leader) {
            my[ind] = ay;
            mi[ind] = ai;
        }
        __syncwarp();
    }
    if (lane == 0) {
        for (int k = 0; k < oversample; ++k) {
            const int dst = n_bins - oversample + k;
            if (dst >= 0 && dst < width) {
                my[dst] = my[1 + k];
                mi[dst] = mi[1 + k];
            }
        }
        double ay = 0.0, ai = 0.0;
        for (int i = 0; i <= n_bins; ++i) {
            ay += my[i];
            my[i] = ay;
            ai += mi[i];
            mi[i] = ai;
        }
    }
    __syncwarp();
    double loc = -INFINITY;
    int ln = 0, ld = 0, ldi = 1 << 30;
    for (int di = 0; di < n_dur; ++di) {
        const int d = (int)dur_bins[di];
        if (d < 1 || d >= n_bins) continue;
        const int m = n_bins - d + 1;
        for (int n = lane; n < m; n += 32) {
            const double y_in = my[n + d] - my[n];
            const double iv_in = mi[n + d] - mi[n];
            const double iv_out = sum_ivar - iv_in;
            if (iv_in < ivar_floor || iv_out < ivar_floor) continue;
            const double yin = y_in / iv_in;
            const double yout = (sum_y - y_in) / iv_out;
            if (yout < yin) continue;
            const double depth = yout - yin;
            const double obj = obj_flag == 0 ? depth / sqrt(1.0 / iv_in + 1.0 / iv_out)
                                             : 0.5 * iv_in * depth * depth;
            if (before(obj, di, n, loc, ldi, ln)) {
                loc = obj;
                ln = n;
                ld = d;
                ldi = di;
            }
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        const double v = __shfl_xor_sync(0xffffffffu, loc, o);
        const int a = __shfl_xor_sync(0xffffffffu, ln, o);
        const int b = __shfl_xor_sync(0xffffffffu, ld, o);
        const int c = __shfl_xor_sync(0xffffffffu, ldi, o);
        if (before(v, c, a, loc, ldi, ln)) {
            loc = v;
            ln = a;
            ld = b;
            ldi = c;
        }
    }
    if (lane != 0) return;
    double* o_power = out;
    double* o_depth = out + n_periods;
    double* o_derr = out + 2 * (int64_t)n_periods;
    double* o_dsnr = out + 3 * (int64_t)n_periods;
    double* o_dur = out + 4 * (int64_t)n_periods;
    double* o_tt = out + 5 * (int64_t)n_periods;
    double* o_ll = out + 6 * (int64_t)n_periods;
    if (!(loc > -INFINITY)) {
        o_power[pidx] = -INFINITY;
        o_depth[pidx] = 0.0;
        o_derr[pidx] = 0.0;
        o_dsnr[pidx] = 0.0;
        o_dur[pidx] = 0.0;
        o_tt[pidx] = 0.0;
        o_ll[pidx] = 0.0;
        return;
    }
    const double y_in = my[ln + ld] - my[ln];
    const double iv_in = mi[ln + ld] - mi[ln];
    const double iv_out = sum_ivar - iv_in;
    const double yin = y_in / iv_in;
    const double yout = (sum_y - y_in) / iv_out;
    const double depth = yout - yin;
    const double derr = sqrt(1.0 / iv_in + 1.0 / iv_out);
    const double dsnr = depth / derr;
    const double ll = 0.5 * iv_in * depth * depth;
    const double dur = (double)ld * bin_duration;
    o_power[pidx] = obj_flag == 0 ? dsnr : ll;
    o_depth[pidx] = depth;
    o_derr[pidx] = derr;
    o_dsnr[pidx] = dsnr;
    o_dur[pidx] = dur;
    o_tt[pidx] = fmod((double)ln * bin_duration + 0.5 * dur, period) + t_min;
    o_ll[pidx] = ll;
}

}  // namespace

extern "C" {

// The unscreened search of one curve over one segment on the GPU: device
// pointers tau (t - t_min), yw (y * ivar), wv (ivar), periods (n_periods),
// dur_bins (n_dur, int64); out: 7 x n_periods FP64, field-major, the numba
// kernel's field order.  Returns 0, a CUDA error code, or -1 when the segment's
// histogram (2 x width doubles) exceeds the device's shared memory.
int oracle_gpu_search(const double* tau, const double* yw, const double* wv, int n_points,
                      const double* periods, int n_periods, const int64_t* dur_bins, int n_dur,
                      double bin_duration, int oversample, int width, double sum_y,
                      double sum_ivar, double t_min, int obj_flag, double ivar_floor, double* out,
                      void* stream) {
    if (n_periods <= 0) return 0;
    const size_t smem = 2 * (size_t)width * sizeof(double);
    int dev = 0, optin = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess)
        e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (e != cudaSuccess) return (int)e;
    if (smem > (size_t)optin) return -1;
    if (smem > 48 * 1024) {
        e = cudaFuncSetAttribute(oracle_period_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem);
        if (e != cudaSuccess) return (int)e;
    }
    oracle_period_kernel<<<n_periods, 32, smem, (cudaStream_t)stream>>>(
        tau, yw, wv, n_points, periods, n_periods, dur_bins, n_dur, bin_duration, oversample,
        width, sum_y, sum_ivar, t_min, obj_flag, ivar_floor, out);
    return (int)cudaGetLastError();
}

}  // extern "C"
