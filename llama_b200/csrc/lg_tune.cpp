// lg_tune.cpp - per-device table of launch parameters (include/lg.h,
// "Launch parameters"): the values the kernels read at launch time, set by
// the caller, by lg_autotune, or loaded from a cache file.
#include <cstdio>
#include <cstring>
#include <mutex>

#include "lg_internal.h"
#include "lg_tune.h"

namespace lg {

namespace {

struct Limits { int64_t lo, hi, def; };

// defaults are the values measured best on B200 for the benchmark
// workloads; lo/hi bound what a kernel accepts
const Limits kLimits[LG_TUNE_COUNT] = {
	{0, 32, 0},         // LG_TUNE_PR_CTAS_PER_SM
	{32, 256, 256},     // LG_TUNE_PPR_KTILE (rounded down to a multiple of 32 dividing K)
	{256, 16384, 2048}, // LG_TUNE_PPR_RANGE
	{256, 16384, 1024}, // LG_TUNE_SSSP_RANGE
	{32, 1u << 20, 512},// LG_TUNE_MS_HEAVY
	{0, 8, 0},          // LG_TUNE_PR_TILE_OCC (0 or 8)
	{0, 1, 0},          // LG_TUNE_SSSP_SPLIT
	{0, 1, 1},          // LG_TUNE_BFS_LEVELS
	{0, 1, 0},          // LG_TUNE_SSSP_LEVELS
};

std::mutex g_mu;
int64_t g_val[LG_TUNE_MAX_DEVICES][LG_TUNE_COUNT];
bool g_init = false;

void init_locked() {
	if (g_init) return;
	for (int d = 0; d < LG_TUNE_MAX_DEVICES; d++)
		for (int k = 0; k < LG_TUNE_COUNT; k++) g_val[d][k] = kLimits[k].def;
	g_init = true;
}

} // namespace

int64_t tune_value(int device, int key) {
	std::lock_guard<std::mutex> lk(g_mu);
	init_locked();
	if (device < 0 || device >= LG_TUNE_MAX_DEVICES || key < 0 || key >= LG_TUNE_COUNT)
		return key >= 0 && key < LG_TUNE_COUNT ? kLimits[key].def : 0;
	return g_val[device][key];
}

} // namespace lg

using namespace lg;

extern "C" lg_status lg_tune_get(int device, int key, int64_t* value) {
	clear_error();
	if (!value) return set_error(LG_EINVAL, "null value");
	if (key < 0 || key >= LG_TUNE_COUNT) return set_error(LG_EINVAL, "unknown tunable %d", key);
	if (device < 0 || device >= LG_TUNE_MAX_DEVICES)
		return set_error(LG_EINVAL, "device %d beyond %d", device, LG_TUNE_MAX_DEVICES);
	*value = tune_value(device, key);
	return LG_OK;
}

extern "C" lg_status lg_tune_set(int device, int key, int64_t value) {
	clear_error();
	if (key < 0 || key >= LG_TUNE_COUNT) return set_error(LG_EINVAL, "unknown tunable %d", key);
	if (device < 0 || device >= LG_TUNE_MAX_DEVICES)
		return set_error(LG_EINVAL, "device %d beyond %d", device, LG_TUNE_MAX_DEVICES);
	if (value < kLimits[key].lo || value > kLimits[key].hi)
		return set_error(LG_EINVAL, "tunable %d: %lld outside [%lld, %lld]", key,
				(long long)value, (long long)kLimits[key].lo, (long long)kLimits[key].hi);
	std::lock_guard<std::mutex> lk(g_mu);
	init_locked();
	g_val[device][key] = value;
	return LG_OK;
}

extern "C" lg_status lg_tune_reset(int device) {
	clear_error();
	if (device < 0 || device >= LG_TUNE_MAX_DEVICES)
		return set_error(LG_EINVAL, "device %d beyond %d", device, LG_TUNE_MAX_DEVICES);
	std::lock_guard<std::mutex> lk(g_mu);
	init_locked();
	for (int k = 0; k < LG_TUNE_COUNT; k++) g_val[device][k] = kLimits[k].def;
	return LG_OK;
}
