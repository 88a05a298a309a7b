// The reference's phase bin of one point, in its own IEEE operations:
//   w = x - P*floor(x/P); ind = int(w/bin) + 1, clipped to [0, width-1]
// (cuPeriod src/cuperiod/methods/_bls_core.py:369-376 / 536-538,
// src/cuperiod/multiband/_bls_joint.py:442-449).  Every operation is rounded on
// its own (no contraction), as the reference's compiled loop does.
#pragma once

namespace blsb200 {

__device__ __forceinline__ int fold_exact(double x, double P, double bin, int width) {
    const double q = __ddiv_rn(x, P);
    const double w = __dsub_rn(x, __dmul_rn(P, floor(q)));
    int ind = (int)__ddiv_rn(w, bin) + 1;
    ind = ind < 0 ? 0 : ind;
    ind = ind > width - 1 ? width - 1 : ind;
    return ind;
}

}  // namespace blsb200
