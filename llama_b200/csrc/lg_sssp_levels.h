// lg_sssp_levels.h - the one-launch form of lg_sssp_delta (lg_sssp_levels.cu).
#ifndef LG_SSSP_LEVELS_H_
#define LG_SSSP_LEVELS_H_

#include "lg_device.cuh"

namespace lg {

// What lg_sssp_delta has set up before its rounds: the views, the initialised
// distances and stamps (sssp_init), the root in q[0], the settled-list
// stamps (split), and the buffers its host loop uses.
struct SsspLevelsArgs {
	SnapCsr out;                 // the rounds' view (the light view under the split)
	SnapCsr heavy;               // the heavy view (split), else == out
	int split;
	uint32_t *q, *qn, *far, *far2;
	uint32_t *dist, *stamp, *fstamp, *bstamp, *blist;
	uint32_t *cnt, *pos;         // V and V + 1 words: a list's slot counts and offsets
	unsigned long long* bsum;    // set by sssp_levels_run
	uint64_t V;
	uint32_t delta, range_max;
};

// Runs the rounds as one cooperative launch; *ran = false (nothing launched)
// when the device has no cooperative launch.  ctl_buf receives the control
// block.  Returns the host loop's rounds, buckets and relaxation count.
lg_status sssp_levels_run(lg_store* s, const SsspLevelsArgs& args, DevBuf& ctl_buf,
		int* rounds, int* buckets, uint64_t* relaxations, bool* ran);

} // namespace lg

#endif // LG_SSSP_LEVELS_H_
