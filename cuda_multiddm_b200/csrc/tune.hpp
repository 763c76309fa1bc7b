// Lag-blocking autotuner: shape keys and the JSON cache (tune.cpp).
#pragma once

#include <string>

#include "../../include/ddm.h"

namespace ddm {

// Key of cfg's shape: frame size and depth, scales, tau list (count, largest, FNV-1a hash),
// chunk and estimator.
std::string tune_key(const ddm_config *cfg);
// The lag_batch_frames (and frames/s) cached for `key` in the file at `path`, if any.
bool tune_lookup(const char *path, const std::string &key, int *lag_batch, double *fps);

}  // namespace ddm
