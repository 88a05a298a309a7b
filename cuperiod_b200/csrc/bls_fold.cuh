// The reference's phase bin of one point.  fold_exact runs its own IEEE
// operations:
//   w = x - P*floor(x/P); ind = int(w/bin) + 1, clipped to [0, width-1]
// (cuPeriod src/cuperiod/methods/_bls_core.py:369-376 / 536-538,
// src/cuperiod/multiband/_bls_joint.py:442-449).  Every operation is rounded on
// its own (no contraction), as the reference's compiled loop does.
#pragma once
#include <stdint.h>

namespace blsb200 {

__device__ __forceinline__ int fold_exact(double x, double P, double bin, int width) {
    const double q = __ddiv_rn(x, P);
    const double w = __dsub_rn(x, __dmul_rn(P, floor(q)));
    int ind = (int)__ddiv_rn(w, bin) + 1;
    ind = ind < 0 ? 0 : ind;
    ind = ind > width - 1 ? width - 1 : ind;
    return ind;
}

// Fast fold: q = x * RN(1/P) rounded onto a 2^-32 grid, then one 32-bit
// multiply-high by S = round(P/bin * 2^fb).  Returns the reference's bin when
// the scaled phase is provably away from every cycle and bin edge (margins mu
// and mphi, derived on the host from the batch's largest time offset), else -1.
__device__ __forceinline__ int fold_fast(double x, double f, uint32_t S, int fb, uint32_t fmask,
                                         uint32_t mu, uint32_t fr_span, uint32_t mphi,
                                         uint32_t phi_span) {
    // x*f + 1.5*2^20 in one rounding: the ulp there is 2^-32, so the low word is
    // round(frac(x*f) * 2^32)
    const double qm = __fma_rn(x, f, 1572864.0);
    const uint32_t phi = (uint32_t)__double2loint(qm);
    const uint32_t v = __umulhi(phi, S);                 // phase * P/bin * 2^fb
    const bool ok = ((phi - mphi) < phi_span) & (((v & fmask) - mu) < fr_span);
    return ok ? (int)(v >> fb) + 1 : -1;
}

// Add v to an int64 kept as a low and a high 32-bit word (add_i64: the
// little-endian words w[0..1]) with two native 32-bit atomics -- the low word,
// then the high word plus the carry out of the low word -- where a 64-bit
// shared atomic would be emulated (sm_100).
// Each add sees the old low word it added to, so every carry is counted once
// and the int64 is the exact sum at any number of adds.
__device__ __forceinline__ void add_i64_split(unsigned* lo_word, unsigned* hi_word, long long v) {
    const unsigned lo = (unsigned)v;
    const unsigned old = atomicAdd(lo_word, lo);
    atomicAdd(hi_word, (unsigned)(v >> 32) + (old + lo < old ? 1u : 0u));
}

__device__ __forceinline__ void add_i64(unsigned* w, long long v) { add_i64_split(w, w + 1, v); }

}  // namespace blsb200
