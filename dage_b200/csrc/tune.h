// tune.h -- the autotuner's cache of launch choices (tile widths), keyed on
// the problem (points per axis, quadrature count, batch) and the device.
// Choices live in the process and, when a cache file is set
// (dage_set_tune_cache or the DAGE_TUNE_CACHE environment variable), are
// read from and appended to that file, so later processes skip the timing.
#pragma once

#include <string>
#include <vector>

namespace dage {

// Key prefix naming the current device (name and SM count): a file shared
// by different GPUs keeps their choices apart.
std::string tune_device_key();
bool tune_lookup(const std::string &key, std::vector<int> &val);
void tune_store(const std::string &key, const std::vector<int> &val);

}  // namespace dage
