// Persistent autotuner choices.
//
// The Dslash variant tuner and the batched-Dslash tuner time their
// candidates on the first call for each (lattice volume, precision, link
// storage, right-hand sides) and keep the fastest for the process.  With
// QPHIX_B200_TUNECACHE=<file> in the environment the choices also go to that
// file, one line per key, and a later process reads them back instead of
// timing again.  Keys carry the GPU's name and SM count, so a file shared
// between machines never hands one GPU another GPU's choices.
#pragma once

#include <string>
#include <vector>

namespace qb {

// true and vals filled when the cache file holds `key`
bool tune_cache_get(const std::string &key, std::vector<double> &vals);
// records key -> vals (appended to the cache file when one is set)
void tune_cache_put(const std::string &key, const std::vector<double> &vals);
// "<GPU name>/<SMs>" of the current device, spaces replaced
std::string tune_device_tag();

}  // namespace qb
