// lg_sssp.cuh - device pieces of delta-stepping SSSP shared by the
// per-round kernels (lg_sssp.cu) and the one-launch form (lg_sssp_levels.cu):
// queue staging, one relaxation round over a queue's slot ranges, the split
// of the far pile at a bucket bound, and the bucket's settled list.
#ifndef LG_SSSP_CUH_
#define LG_SSSP_CUH_

#include "lg_expand.cuh"
#include "lg_queue.cuh"

namespace lg {

constexpr uint32_t kInf = LG_UNREACHED;

// Loads of the near queue / far pile entries: plain (kLd != 1) or through
// L2 (kLd == 1, for buffers rewritten earlier in the same launch).
template <int kLd>
__device__ __forceinline__ uint32_t ld_entry(const uint32_t* p) {
	return kLd == 1 ? __ldcg(p) : *p;
}

// One relaxation round of the calling warp over the queue's slot space
// (pos = exclusive prefix of the queued vertices' slot counts, `total` its
// sum), cut into ranges of at most `range_max` slots and fewer when the
// slots would not give each of the `nwarps` warps one (late rounds queue
// 10^5 - 10^6 vertices with a slot or less each; fixed-size ranges left most
// warps idle while a few walked thousands of entries).  Improved vertices
// below `hi` go to near_next (stamp = round), the others to far (fstamp =
// epoch), through the warp's staging buffers; returns the lane's count of
// successful relaxations.  kLd: how queue and pos are loaded (lg_expand.cuh).
template <int kLd>
__device__ __forceinline__ unsigned long long sssp_relax_ranges(const SnapCsr& out,
		const uint32_t* queue, const uint32_t* pos, uint32_t qlen, uint32_t total,
		uint32_t range_max, uint32_t warp, uint32_t nwarps, uint32_t* dist, uint32_t* stamp,
		uint32_t* fstamp, uint32_t round, uint32_t epoch, uint32_t hi, uint32_t* near_next,
		unsigned long long* near_len, uint32_t* far, unsigned long long* far_len,
		uint32_t* sbuf_near, uint32_t* sbuf_far) {
	uint32_t range = (uint32_t)(((uint64_t)total + nwarps - 1) / nwarps);
	range = min(max((range + 31u) & ~31u, 32u), range_max);
	const uint32_t nranges = (total + range - 1) / range;
	unsigned long long relax = 0;
	uint32_t nn = 0, nf = 0;       // staged near / far appends of this warp
	for (uint32_t r = warp; r < nranges; r += nwarps) {
		range_for_each<kLd>(out, queue, pos, qlen, total, nranges, range, r,
			[&](bool act, uint32_t, uint32_t ov, uint32_t nbr, uint32_t lv, uint32_t idx) {
				bool to_near = false, to_far = false;
				if (act) {
					const uint32_t nd = __ldcg(dist + ov) + __ldg(out.lt->w[lv] + idx);
					if (nd < __ldcg(dist + nbr)) {
						const uint32_t old = atomicMin(dist + nbr, nd);
						relax++;
						if (nd < old) {
							if (nd < hi) to_near = atomicExch(stamp + nbr, round) != round;
							else to_far = atomicExch(fstamp + nbr, epoch) != epoch;
						}
					}
				}
				wq_add(to_near, nbr, sbuf_near, nn, near_next, near_len);
				wq_add(to_far, nbr, sbuf_far, nf, far, far_len);
			});
	}
	wq_flush(sbuf_near, nn, near_next, near_len);
	wq_flush(sbuf_far, nf, far, far_len);
	return relax;
}

// Split of the far pile far[0, n) at bound hi, thread `i0` of `stride`:
// entries with lo <= dist < hi go to the near queue (stamp = round; entries
// below lo were settled from a near queue after they entered the pile),
// entries >= hi are kept (fstamp = epoch); returns the lane's smallest kept
// distance (~0 if none).
template <int kLd>
__device__ __forceinline__ unsigned long long sssp_split_far_body(const uint32_t* far,
		unsigned long long n, const uint32_t* dist, uint32_t* stamp, uint32_t* fstamp,
		uint32_t round, uint32_t epoch, uint32_t lo, uint32_t hi, uint32_t* near,
		unsigned long long* near_len, uint32_t* keep, unsigned long long* keep_len,
		uint32_t* sbuf_near, uint32_t* sbuf_keep, uint64_t i0, uint64_t stride) {
	uint32_t nn = 0, nk = 0;
	unsigned long long m = ~0ull;
	// whole warps loop together (the bound is rounded up to the stride)
	const uint64_t end = (n + 31) & ~31ull;
	for (uint64_t i = i0; i < end; i += stride) {
		uint32_t v = 0, d = kInf;
		if (i < n) { v = ld_entry<kLd>(far + i); d = __ldcg(dist + v); }
		const bool near_take = i < n && d >= lo && d < hi
			&& atomicExch(stamp + v, round) != round;
		const bool keep_take = i < n && d >= hi && d < kInf
			&& atomicExch(fstamp + v, epoch) != epoch;
		wq_add(near_take, v, sbuf_near, nn, near, near_len);
		wq_add(keep_take, v, sbuf_keep, nk, keep, keep_len);
		if (keep_take) m = min(m, (unsigned long long)d);
	}
	wq_flush(sbuf_near, nn, near, near_len);
	wq_flush(sbuf_keep, nk, keep, keep_len);
	return m;
}

// The vertices of the near queue q[0, n) join the bucket's settled list once
// each (bstamp = bucket), counted in *len; thread `i0` of `stride`.
template <int kLd>
__device__ __forceinline__ void sssp_collect_body(const uint32_t* q, uint32_t n,
		uint32_t* bstamp, uint32_t bucket, uint32_t* blist, unsigned long long* len,
		uint32_t* sbuf, uint64_t i0, uint64_t stride) {
	uint32_t nn = 0;
	const uint64_t end = ((uint64_t)n + 31) & ~31ull;
	for (uint64_t i = i0; i < end; i += stride) {
		const uint32_t v = i < n ? ld_entry<kLd>(q + i) : 0u;
		const bool take = i < n && atomicExch(bstamp + v, bucket) != bucket;
		wq_add(take, v, sbuf, nn, blist, len);
	}
	wq_flush(sbuf, nn, blist, len);
}

} // namespace lg

#endif // LG_SSSP_CUH_
