// Host-side builder of the reference's default BLS trial grid (bls_grid.cpp).
#pragma once
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/bls_b200.h"

namespace blsb200 {

struct DefaultGrid {
    std::vector<double> periods;        // ascending within each segment
    std::vector<int64_t> seg_offsets;   // n_segments + 1 offsets into periods
    std::vector<int32_t> seg_start;     // per segment: its index k among the segment starts
};

// The default grid of one baseline; BLS_OK, or an error code with `err` set.
int build_default_grid(const BlsDefaultGrid& spec, double baseline, DefaultGrid& out,
                       std::string& err);
// Its number of periods, or -1 when it cannot be built.
int64_t default_grid_size(const BlsDefaultGrid& spec, double baseline);

}  // namespace blsb200
