// Autotuner: shape keys and the JSON cache (tune.cpp).
#pragma once

#include <string>

#include "../../include/ddm.h"

namespace ddm {

// Key of cfg's shape: frame size and depth, scales, tau list (count, largest, FNV-1a hash),
// chunk, estimator and the small-tile DFT choice.
std::string tune_key(const ddm_config *cfg);
// The tuned values cached for `key` in the file at `path`, if any.
struct TunedValues {
    int lag_batch = 0, lag_geometry = 0, fft_group = 0, fft_per_tile = 0;
    double fps = 0.0;
};
bool tune_lookup(const char *path, const std::string &key, TunedValues *out);

}  // namespace ddm
