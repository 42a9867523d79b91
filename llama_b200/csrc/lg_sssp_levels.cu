// lg_sssp_levels.cu - delta-stepping SSSP in one cooperative launch.
//
// lg_sssp_delta's host loop reads the step's counters back after every
// relaxation round, bucket split and heavy phase (about 70-90 per root on an
// R-MAT scale-24 snapshot, each a launch sequence and a host round trip).
// sssp_levels runs the same steps inside one grid of co-resident CTAs and
// replaces the round trips by grid barriers (lg_coop.cuh): every CTA reads
// the previous step's counters after the barrier and applies the host loop's
// rules, so the steps, their order and the distances equal the loop's.
//
// Steps (the host loop's, lg_sssp.cu):
//   relax   the near queue's vertices relax their edges (the light view under
//           LG_TUNE_SSSP_SPLIT, whose rounds also add the queue to the
//           bucket's settled list); improved vertices below the bucket bound
//           form the next near queue, the others join the far pile;
//   heavy   (split only) when the near queue drains, the bucket's settled
//           vertices relax their heavy edges once, into the far pile;
//   split   when both drain, the far pile is split at the next bound; if
//           nothing falls below it, a second split at the bucket of the
//           smallest distance left.
// A relax or heavy step forms its list's slot offsets like the one-launch
// BFS: every CTA in its own shared memory for at most 2048 entries (no
// barrier), else per-CTA sums and offsets in two barrier-separated phases.
// Counters rotate over three slots and count appends only (zeroed two steps
// ahead); each CTA adds them to the lengths it keeps, so the far pile's and
// the settled list's appends go after their current ends.
#include "lg_coop.cuh"
#include "lg_expand.cuh"
#include "lg_sssp.cuh"
#include "lg_sssp_levels.h"

#include <mutex>

namespace lg {

namespace {

constexpr int kSlThreads = 512;
constexpr int kSlWarps = kSlThreads / 32;
constexpr int kSlSmallPer = 4;          // queue entries per thread of the barrier-free scan

enum SlStep : int { kStepNone = 0, kStepRelax, kStepHeavy, kStepSplit };

// Control block (device memory; bfs-style reset by sssp_levels_init).
struct SlCtl {
	unsigned long long ctr[3][4];   // per step: [0] near appends, [1] far appends,
	                                // [2] relaxations (split: max of ~kept distance),
	                                // [3] settled-list appends
	CoopBar bar;                    // err bit 1: slots above 2^32, bit 2: a count out
	                                // of range, bit 3: step cap
	int32_t rounds, buckets;
	unsigned long long relaxations;
};

__global__ void sssp_levels_init(SlCtl* c) {
	if (blockIdx.x == 0 && threadIdx.x == 0) {
		for (int i = 0; i < 3; i++)
			for (int j = 0; j < 4; j++) c->ctr[i][j] = 0;
		c->bar.count = 0;
		c->bar.err = 0;
		c->rounds = c->buckets = 0;
		c->relaxations = 0;
	}
}

// Slot offsets of list[0, n) over view g into pos (or, for a small list, the
// CTA's s_pos); returns the slot total in *total and whether s_pos holds
// them.  false if a barrier failed or the total passed 2^32 (err set).
__device__ bool list_offsets(const SnapCsr& g, const uint32_t* list, uint32_t n, uint32_t* cnt,
		uint32_t* pos, unsigned long long* bsum, uint32_t* s_pos, SlCtl* c, uint32_t* total,
		bool* small) {
	const uint32_t tid = threadIdx.x;
	*small = n <= (uint32_t)(kSlThreads * kSlSmallPer);
	if (*small) {
		uint32_t kc[kSlSmallPer];
		unsigned long long sum = 0;
#pragma unroll
		for (int j = 0; j < kSlSmallPer; j++) {
			const uint32_t i = tid * kSlSmallPer + j;
			uint32_t f0;
			kc[j] = i < n ? vertex_slots(g, __ldcg(list + i), &f0) : 0u;
			sum += kc[j];
		}
		if (block_sum<kSlWarps>(sum) >= (1ull << 32)) {
			if (tid == 0) atomicOr(&c->bar.err, 2u);
			return false;                    // every CTA sees the same total
		}
		uint32_t all;
		uint32_t ex = block_exclusive_scan<kSlWarps>((uint32_t)sum, &all);
#pragma unroll
		for (int j = 0; j < kSlSmallPer; j++) {
			const uint32_t i = tid * kSlSmallPer + j;
			if (i < n) s_pos[i] = ex;
			ex += kc[j];
		}
		if (tid == 0) s_pos[n] = all;
		*total = all;
		__syncthreads();
		return true;
	}
	// phase A: slot counts of this CTA's share, per-CTA sums
	const uint32_t chunk = (n + gridDim.x - 1u) / gridDim.x;
	const uint32_t c0 = min(n, blockIdx.x * chunk), c1 = min(n, c0 + chunk);
	unsigned long long s = 0;
	for (uint32_t i = c0 + tid; i < c1; i += blockDim.x) {
		uint32_t f0;
		const uint32_t k = vertex_slots(g, __ldcg(list + i), &f0);
		cnt[i] = k;
		s += k;
	}
	s = block_sum<kSlWarps>(s);
	if (tid == 0) bsum[blockIdx.x] = s;
	if (!grid_barrier(&c->bar)) return false;
	// phase B: offsets (every CTA forms the same total)
	unsigned long long pre = 0, tot = 0;
	for (uint32_t b = tid; b < gridDim.x; b += blockDim.x) {
		const unsigned long long x = __ldcg(bsum + b);
		tot += x;
		if (b < blockIdx.x) pre += x;
	}
	pre = block_sum<kSlWarps>(pre);
	tot = block_sum<kSlWarps>(tot);
	if (tot >= (1ull << 32)) {
		if (tid == 0) atomicOr(&c->bar.err, 2u);
		return false;
	}
	uint32_t run = (uint32_t)pre;
	for (uint32_t p = c0; p < c1; p += blockDim.x) {
		const uint32_t i = p + tid;
		const uint32_t x = i < c1 ? __ldcg(cnt + i) : 0u;
		uint32_t piece;
		const uint32_t ex = block_exclusive_scan<kSlWarps>(x, &piece);
		if (i < c1) pos[i] = run + ex;
		run += piece;
	}
	if (blockIdx.x == gridDim.x - 1u && tid == 0) pos[n] = (uint32_t)tot;
	*total = (uint32_t)tot;
	return grid_barrier(&c->bar);
}

// One relaxation step, kept out of line so that its register allocation is
// its own (inlined into the kernel's state machine it spilled in the loop).
__device__ __noinline__ unsigned long long relax_step(const SnapCsr& g, const uint32_t* list,
		const uint32_t* pos, uint32_t n, uint32_t total, uint32_t range_max, uint32_t gwarp,
		uint32_t nwarps, uint32_t* dist, uint32_t* stamp, uint32_t* fstamp, uint32_t round,
		uint32_t epoch, uint32_t hi, uint32_t* qn, unsigned long long* nxt, uint32_t* far_end,
		uint32_t* sbuf_near, uint32_t* sbuf_far) {
	return sssp_relax_ranges<2>(g, list, pos, n, total, range_max, gwarp, nwarps, dist, stamp,
			fstamp, round, epoch, hi, qn, nxt, far_end, nxt + 1, sbuf_near, sbuf_far);
}

// Two CTAs of 512 per SM.
__global__ void __launch_bounds__(kSlThreads, 2)
sssp_levels(SsspLevelsArgs a, SlCtl* c) {
	__shared__ uint32_t sbuf[kSlWarps][2][kPushBuf];
	__shared__ uint32_t s_pos[kSlThreads * kSlSmallPer + 1];
	const uint32_t tid = threadIdx.x, lane = tid & 31u, wid = tid >> 5;
	const uint32_t gtid = blockIdx.x * blockDim.x + tid;
	const uint32_t nthreads = gridDim.x * blockDim.x;
	const uint32_t nwarps = nthreads >> 5, gwarp = gtid >> 5;
	uint32_t *q = a.q, *qn = a.qn, *far = a.far, *far2 = a.far2;
	// every CTA keeps the same copy of the traversal state (the host loop's)
	unsigned long long qlen = 1, flen = 0, blen = 0, relaxations = 0;
	uint32_t lo = 0, hi = a.delta, round = 0, epoch = 0, bid = 0;
	int32_t buckets = 1, attempt = 0;
	int last = kStepNone;
	const unsigned long long step_cap = 4ull * a.V + 64;
	for (unsigned long long step = 0;; step++) {
		unsigned long long* res = c->ctr[step % 3];          // the last step's counts
		unsigned long long* nxt = c->ctr[(step + 1) % 3];
		// apply the last step's counts
		bool retry = false;
		if (last == kStepRelax) {
			const unsigned long long nq = __ldcg(res + 0), nf = __ldcg(res + 1);
			if (nq > a.V || flen + nf > a.V || blen + __ldcg(res + 3) > a.V) {
				if (tid == 0) atomicOr(&c->bar.err, 4u);
				return;
			}
			qlen = nq;
			flen += nf;
			relaxations += __ldcg(res + 2);
			if (a.split) blen += __ldcg(res + 3);
			uint32_t* t = q; q = qn; qn = t;
		} else if (last == kStepHeavy) {
			const unsigned long long nf = __ldcg(res + 1);
			if (__ldcg(res + 0) != 0 || flen + nf > a.V) {
				if (tid == 0) atomicOr(&c->bar.err, 4u);
				return;
			}
			flen += nf;
			relaxations += __ldcg(res + 2);
			blen = 0;
			bid++;
		} else if (last == kStepSplit) {
			const unsigned long long nq = __ldcg(res + 0), nk = __ldcg(res + 1);
			if (nq > a.V || nk > a.V) {
				if (tid == 0) atomicOr(&c->bar.err, 4u);
				return;
			}
			qlen = nq;
			flen = nk;
			uint32_t* t = far; far = far2; far2 = t;
			buckets++;
			if (attempt == 0 && qlen == 0 && flen > 0) {
				// nothing below the bound: jump to the bucket of the smallest
				// distance left and split again
				const uint32_t mind = (uint32_t)~__ldcg(res + 2);
				lo = (mind / a.delta) * a.delta;
				hi = (lo > kInf - a.delta) ? kInf : lo + a.delta;
				retry = true;
			}
		}
		if (blockIdx.x == 0 && tid < 4) c->ctr[(step + 2) % 3][tid] = 0;
		if (qlen == 0 && flen == 0 && blen == 0) break;
		if (step >= step_cap) {
			if (tid == 0) atomicOr(&c->bar.err, 8u);
			return;
		}

		if (qlen > 0 || blen > 0) {
			// relax: the near queue (over the light view under the split); or,
			// when the bucket drained, heavy: its settled vertices' heavy edges
			const bool heavy_step = qlen == 0;
			round++;
			last = heavy_step ? kStepHeavy : kStepRelax;
			const SnapCsr g = heavy_step ? a.heavy : a.out;
			const uint32_t* list = heavy_step ? a.blist : q;
			const uint32_t n = (uint32_t)(heavy_step ? blen : qlen);
			if (a.split && !heavy_step)
				sssp_collect_body<1>(q, n, a.bstamp, bid, a.blist + blen, nxt + 3, sbuf[wid][0],
						gtid, nthreads);
			uint32_t total;
			bool small;
			if (!list_offsets(g, list, n, a.cnt, a.pos, a.bsum, s_pos, c, &total, &small))
				return;
			// plain loads: shared offsets, or global ones written before a barrier
			unsigned long long r = relax_step(g, list, small ? s_pos : a.pos, n, total,
					a.range_max, gwarp, nwarps, a.dist, a.stamp, a.fstamp, round, epoch, hi, qn,
					nxt, far + flen, sbuf[wid][0], sbuf[wid][1]);
			r = block_sum<kSlWarps>(r);
			if (tid == 0 && r) atomicAdd(nxt + 2, r);
		} else {
			// both drained: split the far pile at the next bound (or, on a
			// retry, at the bucket of the smallest distance left)
			if (retry) {
				attempt = 1;
			} else {
				lo = hi;
				hi = (hi > kInf - a.delta) ? kInf : hi + a.delta;
				attempt = 0;
			}
			round++;
			epoch++;
			last = kStepSplit;
			const unsigned long long m = sssp_split_far_body<1>(far, flen, a.dist, a.stamp,
					a.fstamp, round, epoch, lo, hi, q, nxt, far2, nxt + 1, sbuf[wid][0],
					sbuf[wid][1], gtid, nthreads);
			unsigned long long mm = m;
#pragma unroll
			for (int o = 16; o > 0; o >>= 1) mm = min(mm, __shfl_down_sync(0xffffffffu, mm, o));
			if (lane == 0 && mm != ~0ull) atomicMax(nxt + 2, ~mm);
		}
		if (!grid_barrier(&c->bar)) return;
	}
	if (blockIdx.x == 0 && tid == 0) {
		c->rounds = (int32_t)round;
		c->buckets = buckets;
		c->relaxations = relaxations;
	}
}

std::mutex g_coop_mu;
int g_coop[LG_TUNE_MAX_DEVICES];          // co-resident CTAs + 1, 0 = not probed

int coop_grid(int device) {
	std::lock_guard<std::mutex> lk(g_coop_mu);
	if (device < 0 || device >= LG_TUNE_MAX_DEVICES) return 0;
	if (!g_coop[device])
		g_coop[device] = 1 + coop_grid_size((const void*)sssp_levels, kSlThreads, device);
	return g_coop[device] - 1;
}

} // namespace

lg_status sssp_levels_run(lg_store* s, const SsspLevelsArgs& args, DevBuf& ctl_buf,
		int* rounds, int* buckets, uint64_t* relaxations, bool* ran) {
	*ran = false;
	const int grid = coop_grid(s->device);
	if (grid <= 0) return LG_OK;
	cudaStream_t st = s->stream;
	LG_TRY(ctl_buf.reserve(sizeof(SlCtl) + (size_t)grid * sizeof(unsigned long long)));
	SlCtl* ctl = ctl_buf.as<SlCtl>();
	SsspLevelsArgs a = args;
	a.bsum = reinterpret_cast<unsigned long long*>(ctl_buf.as<unsigned char>() + sizeof(SlCtl));
	sssp_levels_init<<<1, 32, 0, st>>>(ctl);
	LG_CUDA(cudaGetLastError(), "sssp_levels_init");
	void* kargs[] = {&a, &ctl};
	LG_CUDA(cudaLaunchCooperativeKernel((const void*)sssp_levels, dim3((unsigned)grid),
			dim3(kSlThreads), kargs, 0, st), "sssp_levels");
	s->launches += 2;
	SlCtl h;
	LG_CUDA(cudaMemcpyAsync(&h, ctl, sizeof(h), cudaMemcpyDeviceToHost, st), "d2h");
	LG_CUDA(cudaStreamSynchronize(st), "sssp_levels");
	s->d2h_bytes += sizeof(h);
	if (h.bar.err & 1u) return set_error(LG_ETIMEOUT, "sssp: a grid barrier wait ran out");
	if (h.bar.err & 2u) return set_error(LG_ENOTSUP, "sssp: a queue holds 2^32 or more slots");
	if (h.bar.err & 4u) return set_error(LG_ECUDA, "sssp: a queue count out of range");
	if (h.bar.err & 8u) return set_error(LG_ECUDA, "sssp: step cap reached");
	*rounds = h.rounds;
	*buckets = h.buckets;
	*relaxations = h.relaxations;
	*ran = true;
	return LG_OK;
}

} // namespace lg
