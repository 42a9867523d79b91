// lg_expand.cuh - load-balanced expansion of a vertex list over a snapshot.
//
// A list of vertices (all vertices in order, or a BFS/SSSP frontier) owns a
// virtual slot space: entry i covers slots [pos[i], pos[i+1]) where pos is the
// exclusive prefix of the entries' fragment lengths.  That space is cut into
// ranges of a fixed number of slots and every warp processes whole ranges,
// so a vertex with 10^5 in-edges is spread over many warps instead of
// stalling one, and every warp does the same amount of work.
//
// Inside a range the warp takes up to 32 entries at a time (lane j holds
// entry j of the window: its vertex, its first fragment and its slot span
// clipped to the range) and walks the window's slots 32 x kUnroll at a time:
// lane k of a chunk owns slot base + k; the owning entry is the last lane
// whose clipped span starts at or before that slot (5 shuffles), and the
// fragment holding it is found by skipping whole fragments of that vertex
// (at most one per level).  All loads of the kUnroll chunks are issued before
// any of them is used, which keeps kUnroll x 32 gathers in flight per warp.
#ifndef LG_EXPAND_CUH_
#define LG_EXPAND_CUH_

#include "lg_device.cuh"

namespace lg {

constexpr int kUnroll = 4;

// Loads of the list and its offsets (kLd): 0 = through the read-only path
// (the default); 1 = through L2, for a kernel that rewrites them between its
// own phases (the read-only path may hold lines from before the rewrite);
// 2 = plain generic loads, for offsets kept in shared memory.
template <int kLd>
__device__ __forceinline__ uint32_t ld_list(const uint32_t* p) {
	if (kLd == 0) return __ldg(p);
	if (kLd == 1) return __ldcg(p);
	return *p;
}

// First index e in [0, m] with arr[e] >= x (arr sorted, arr[m] the total),
// computed by the whole warp with 32-way probing.
template <int kLd = 0>
__device__ __forceinline__ uint32_t warp_lower_bound(const uint32_t* arr, uint32_t m,
		uint32_t x) {
	const uint32_t lane = threadIdx.x & 31u;
	uint32_t lo = 0, hi = m;                 // answer in [lo, hi]
	while (hi - lo > 32) {
		const uint32_t step = (hi - lo + 31) / 32;
		uint32_t p = lo + lane * step;
		bool below = p < hi && ld_list<kLd>(arr + p) < x;
		unsigned b = __ballot_sync(0xffffffffu, below);
		uint32_t c = __popc(b);              // probes below x: lanes 0..c-1
		uint32_t nlo = c ? lo + (c - 1) * step + 1 : lo;
		uint32_t nhi = lo + c * step;
		if (nhi > hi) nhi = hi;
		lo = nlo;
		hi = nhi;
	}
	uint32_t p = lo + lane;
	bool below = p < hi && ld_list<kLd>(arr + p) < x;
	return lo + __popc(__ballot_sync(0xffffffffu, below));
}

// One window of up to 32 list entries inside a range [a, b).
struct Window {
	uint32_t e;        // entry index of this lane
	bool valid;        // lane holds an entry
	uint32_t v;        // its vertex
	uint32_t f0;       // its first fragment
	uint32_t start;    // pos[e], start of the entry's full slot span
	uint32_t s0, s1;   // its span clipped to the range
	uint32_t lo, hi;   // slots covered by the whole window
};

template <int kLd = 0>
__device__ __forceinline__ Window load_window(const SnapCsr& g, const uint32_t* list,
		const uint32_t* pos, uint32_t ew, uint32_t e_end, uint32_t a, uint32_t b) {
	const uint32_t lane = threadIdx.x & 31u;
	Window w;
	w.e = ew + lane;
	w.valid = w.e < e_end;
	w.v = 0; w.f0 = 0; w.start = 0; w.s0 = 0; w.s1 = 0;
	if (w.valid) {
		w.v = list ? ld_list<kLd>(list + w.e) : w.e;
		w.f0 = __ldg(g.frag_off + w.v);
		w.start = ld_list<kLd>(pos + w.e);
		const uint32_t end = ld_list<kLd>(pos + w.e + 1);
		w.s0 = max(w.start, a);
		w.s1 = min(end, b);
		if (w.s1 < w.s0) w.s1 = w.s0;
	}
	// invalid lanes sit at the end of the window with an empty span
	uint32_t last_s1 = w.s1;
	const unsigned vm = __ballot_sync(0xffffffffu, w.valid);
	const int last = 31 - __clz(vm);
	last_s1 = __shfl_sync(0xffffffffu, w.s1, last);
	if (!w.valid) { w.s0 = last_s1; w.s1 = last_s1; }
	w.lo = __shfl_sync(0xffffffffu, w.s0, 0);
	w.hi = last_s1;
	return w;
}

// Slot k of the window: owner lane, and the (level, index) it maps to.
__device__ __forceinline__ void locate_slot(const SnapCsr& g, const Window& w,
		uint32_t k, uint32_t* owner, uint32_t* lv, uint32_t* idx) {
	uint32_t o = 0;
#pragma unroll
	for (uint32_t step = 16; step > 0; step >>= 1) {
		const uint32_t cand = o + step;
		const uint32_t s = __shfl_sync(0xffffffffu, w.s0, cand);
		if (s <= k) o = cand;
	}
	// lanes with equal s0 (empty spans) resolve to the last one, whose span
	// holds k
	const uint32_t ostart = __shfl_sync(0xffffffffu, w.start, o);
	uint32_t f = __shfl_sync(0xffffffffu, w.f0, o);
	*owner = o;
	if (k < w.hi) {
		uint32_t r = k - ostart;
		uint2 fr = g.frags[f];
		while (r >= frag_len(fr)) { r -= frag_len(fr); fr = g.frags[++f]; }
		*lv = frag_level(fr);
		*idx = fr.x + r;
	} else {
		*lv = 0;
		*idx = 0;
	}
}

// Entries of range [a, b): e_begin includes an entry that started before a
// and reaches into the range; e_end stops before entries starting at or
// after b (for the last range, b covers the whole list).
template <int kLd = 0>
__device__ __forceinline__ void range_entries(const uint32_t* pos, uint32_t n,
		uint32_t a, uint32_t b, bool last_range, uint32_t* e_begin, uint32_t* e_end) {
	uint32_t eb = warp_lower_bound<kLd>(pos, n, a);
	if (eb > 0 && (eb == n || ld_list<kLd>(pos + eb) > a)) {
		// the entry before eb may straddle a
		if (ld_list<kLd>(pos + eb) > a || eb == n) eb--;
	}
	*e_begin = eb;
	*e_end = last_range ? n : warp_lower_bound<kLd>(pos, n, b);
}

// Process range `r` of a list's slot space (ranges of `range` slots, nranges
// of them, `total` slots) and call, for every chunk of 32 slots and on all 32
// lanes, body(active, owner_lane, owner_vertex, nbr, level, index) - active =
// the lane holds a live slot.  The body may use warp collectives.  Owner
// lanes are non-decreasing across a chunk and lanes past the window's last
// slot get owner lane 31, so owner_lane is a safe key for segmented
// reductions (owner_vertex of such lanes is a placeholder).
template <int kLd = 0, class Body>
__device__ __forceinline__ void range_for_each(const SnapCsr& g, const uint32_t* list,
		const uint32_t* pos, uint32_t n, uint32_t total, uint32_t nranges,
		uint32_t range, uint32_t r, Body&& body) {
	const uint32_t lane = threadIdx.x & 31u;
	const bool last_range = r == nranges - 1;
	const uint32_t ra = r * range;
	const uint32_t rb = last_range ? total : min(total, ra + range);
	uint32_t e_begin, e_end;
	range_entries<kLd>(pos, n, ra, rb, last_range, &e_begin, &e_end);
	const LevelTab* lt = g.lt;
	for (uint32_t ew = e_begin; ew < e_end; ew += 32) {
		const Window w = load_window<kLd>(g, list, pos, ew, e_end, ra, rb);
		for (uint32_t base = w.lo; base < w.hi; base += 32 * kUnroll) {
			uint32_t nb[kUnroll], own[kUnroll], lvs[kUnroll], ids[kUnroll];
			bool act[kUnroll];
#pragma unroll
			for (int u = 0; u < kUnroll; u++) {
				const uint32_t k = base + u * 32 + lane;
				locate_slot(g, w, k, &own[u], &lvs[u], &ids[u]);
				act[u] = k < w.hi;
				nb[u] = 0;
				if (act[u]) {
					const uint32_t word = __ldg(lt->del[lvs[u]] + (ids[u] >> 5));
					nb[u] = __ldg(lt->ids[lvs[u]] + ids[u]);
					act[u] = !((word >> (ids[u] & 31)) & 1u);
				}
			}
#pragma unroll
			for (int u = 0; u < kUnroll; u++) {
				const uint32_t ov = __shfl_sync(0xffffffffu, w.v, own[u]);
				body(act[u], own[u], ov, nb[u], lvs[u], ids[u]);
			}
		}
	}
	(void)lane;
}

// Frontier bookkeeping shared by the list-driven kernels: per-entry slot
// counts, to be scanned into the `pos` offsets range_for_each expects.
static __global__ void list_slots(SnapCsr g, const uint32_t* list, uint32_t n,
		uint32_t* cnt) {
	const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	uint32_t f0;
	cnt[i] = vertex_slots(g, list ? __ldg(list + i) : (uint32_t)i, &f0);
}

} // namespace lg

#endif // LG_EXPAND_CUH_
