// Cache of batch configurations chosen by cctagb_autotune: a JSON file
// {"version": V, "entries": {key: {"batchWaveFrames": .., "identLayout": ..,
// "ms_per_frame": ..}}}, keyed by GPU, frame size, frames per call and crowns.
// Host only (no CUDA).
#pragma once

#include <string>

#include "cctag_b200.h"

namespace cctagb {
namespace tune {

constexpr int kCacheVersion = 2;

std::string key(const char* gpu_name, int sm_count, int w, int h, int frames, int n_crowns);
// Frames of several sizes: named by their total pixel count.
std::string key_mixed(const char* gpu_name, int sm_count, long long total_px, int frames, int n_crowns);
// True and *out filled (from_cache = 1) when the file holds the key.
bool cache_get(const std::string& path, const std::string& key, cctagb_tune_choice& out);
// Adds or replaces the key's entry; throws Error when the file cannot be written.
void cache_put(const std::string& path, const std::string& key, const cctagb_tune_choice& c);

}  // namespace tune
}  // namespace cctagb
