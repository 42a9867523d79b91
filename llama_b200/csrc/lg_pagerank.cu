// lg_pagerank.cu - PageRank, pull direction, FP64, over a snapshot's in-CSR.
//
// Reference: ll_b_pagerank_pull_ext<Graph,double>::run
// (benchmark/benchmarks/pagerank.h:98-182): pr0 = 1/N (N = max_nodes),
// then `max` times  pr'[t] = (1-d)/N + d * sum_{w in in(t)} pr[w]/out_degree(w),
// dangling mass dropped.
//
// Instead of gathering pr[w] and out_degree(w) per edge (two dependent random
// loads in the reference), each iteration writes contrib'[t] = pr'[t] /
// out_degree(t), so an edge costs one 4-byte id load and one 8-byte gather.
// The division is the one the reference performs per edge, so the gathered
// values are bit-identical; only the order in which a vertex's values are
// added differs from the reference's left-to-right loop (FP64, well within
// 1e-12 in every case), and it is fixed, so results are deterministic.
//
// lg_pagerank_pull first flattens the snapshot's live in-adjacency once per
// call (flat_count / flat_write: the virtual slot space of the in-CSR in
// vertex order, each vertex's fragments newest first, deleted slots
// dropped), then runs every iteration over that flat edge array:
//
//   flat ids    E x u32      in-neighbour of every live in-edge
//   heads       bit per edge set where a vertex's in-edges begin
//   nz_rows     R x u32      the vertices with in-edges, in order
//   nz_off      R x u32      where each of them begins in the flat array
//   tile_seg    per tile     heads before the tile's first edge
//
// pr_flat_step gives each warp a tile of kFlatTile consecutive edges, 8 per
// lane: it issues the tile's id loads and gathers up front, adds each
// lane's values serially and joins the lanes with one segmented warp scan
// keyed by the head bits; a vertex that runs past a tile boundary leaves
// partials (carry_first, carry_last) that pr_flat_fixup adds.  No block
// barriers: each warp stages its finished row sums in its own shared memory.
// Vertices without in-edges have the constant rank (1-d)/N after the first
// iteration and are written once (pr_empty_rows).
//
// lg_pagerank_pull_noalloc cannot hold the E-sized flat array, so it walks
// the fragments directly every iteration (pr_pull_step, one CTA per 1024
// virtual slots, values staged in shared memory).
#include "lg_device.cuh"
#include "lg_expand.cuh"

#include <mutex>

namespace lg {

constexpr int kPrThreads = 128;
constexpr int kPrPerThread = 8;
constexpr uint32_t kPrRange = kPrThreads * kPrPerThread;        // 1024 slots
static_assert(kPrRange == kBlockSlots, "range_lb is computed for kBlockSlots");
constexpr uint32_t kPrMaxFrags = kPrRange + 2 * LG_MAX_LEVELS;   // fragments touching a block
constexpr uint32_t kPrLong = 64;       // entries with more slots are reduced by a warp

// The in-CSR virtual slot space of a snapshot cut into kPrRange-slot blocks.
struct SlotSpace {
	SnapCsr in;
	const uint32_t* pos;       // V + 1 in-CSR slot prefix
	const uint32_t* range_lb;  // nranges + 1 block entry bounds
	uint32_t total;            // pos[V]
	uint32_t nranges;
};

// Shared-memory map from the slots of one block to their fragments.
struct BlockMap {
	uint2 ftab[kPrMaxFrags];           // fragments of the block's entries
	uint32_t fstart[kPrMaxFrags + 1];  // their absolute virtual starts
	uint32_t fidx[kPrRange];           // block slot -> index into ftab
	uint32_t wsum[kPrThreads / 32];
	uint32_t eb, ee, nf;               // block entries [eb, ee), fragments
};

// Builds m for block r (slots [ra, rb)); every thread of the block calls it
// and it returns synchronised.
__device__ void map_block(const SlotSpace& sp, uint32_t r, uint32_t ra, uint32_t rb,
		BlockMap& m) {
	const uint32_t tid = threadIdx.x, lane = tid & 31u, wid = tid >> 5;
	const bool last_range = r == sp.nranges - 1;
	const uint32_t V = (uint32_t)sp.in.V;
	if (tid == 0) {
		// entries of the block: those starting in [ra, rb), plus the one
		// straddling ra (precomputed lower bounds, see block_lower_bounds)
		uint32_t eb = __ldg(sp.range_lb + r);
		if (eb > 0 && (eb == V || __ldg(sp.pos + eb) > ra)) eb--;
		m.eb = eb;
		m.ee = last_range ? V : __ldg(sp.range_lb + r + 1);
	}
	__syncthreads();
	const uint32_t eb = m.eb, ee = m.ee;

	// fragment table of the block's entries, with absolute virtual starts
	const uint32_t f_begin = __ldg(sp.in.frag_off + eb);
	uint32_t nf = (ee > eb) ? __ldg(sp.in.frag_off + ee) - f_begin : 0;
	// every fragment of an entry inside the block has a slot in the block,
	// and only the two end entries add others, so nf <= kPrMaxFrags
	if (nf > kPrMaxFrags) nf = kPrMaxFrags;
	const uint32_t vbase = __ldg(sp.pos + eb);
	uint32_t carry = 0;
	for (uint32_t c0 = 0; c0 < nf; c0 += kPrThreads) {
		const uint32_t i = c0 + tid;
		uint32_t len = 0;
		if (i < nf) { const uint2 fr = sp.in.frags[f_begin + i]; m.ftab[i] = fr; len = frag_len(fr); }
		// block exclusive scan of len
		uint32_t x = len;
#pragma unroll
		for (int o = 1; o < 32; o <<= 1) {
			const uint32_t t = __shfl_up_sync(0xffffffffu, x, o);
			if (lane >= (uint32_t)o) x += t;
		}
		if (lane == 31) m.wsum[wid] = x;
		__syncthreads();
		uint32_t before = carry;
		for (uint32_t w2 = 0; w2 < wid; w2++) before += m.wsum[w2];
		if (i < nf) m.fstart[i] = vbase + before + x - len;
		uint32_t tot = 0;
		for (uint32_t w2 = 0; w2 < kPrThreads / 32; w2++) tot += m.wsum[w2];
		carry += tot;
		__syncthreads();
	}
	if (tid == 0) { m.fstart[nf] = vbase + carry; m.nf = nf; }
	// slot -> fragment map: each fragment marks the first block slot it
	// covers (the last of the fragments starting at or before ra marks slot
	// 0), then an inclusive max-scan over the block's slots spreads the marks
	for (uint32_t k = tid; k < kPrRange; k += kPrThreads) m.fidx[k] = 0;
	__syncthreads();
	for (uint32_t i = tid; i < nf; i += kPrThreads) {
		const uint32_t st = m.fstart[i];
		if (st < rb) atomicMax(&m.fidx[st > ra ? st - ra : 0], i);
	}
	__syncthreads();
	{
		// thread t scans slots [8t, 8t + 8) serially, then a block scan of
		// the thread maxima carries the mark across threads
		uint32_t mx = 0, loc[kPrPerThread];
#pragma unroll
		for (int u = 0; u < kPrPerThread; u++) {
			mx = max(mx, m.fidx[tid * kPrPerThread + u]);
			loc[u] = mx;
		}
		uint32_t x = mx;
#pragma unroll
		for (int o = 1; o < 32; o <<= 1) {
			const uint32_t t = __shfl_up_sync(0xffffffffu, x, o);
			if (lane >= (uint32_t)o) x = max(x, t);
		}
		if (lane == 31) m.wsum[wid] = x;
		__syncthreads();
		uint32_t before = __shfl_up_sync(0xffffffffu, x, 1);
		if (lane == 0) before = 0;
		for (uint32_t w2 = 0; w2 < wid; w2++) before = max(before, m.wsum[w2]);
#pragma unroll
		for (int u = 0; u < kPrPerThread; u++)
			m.fidx[tid * kPrPerThread + u] = max(before, loc[u]);
	}
	__syncthreads();
}

// Level and in-level index of block slot k (virtual slot ra + k); false if
// the block has no such slot.
__device__ __forceinline__ bool block_slot(const BlockMap& m, uint32_t ra, uint32_t rb,
		uint32_t k, uint32_t* lv, uint32_t* idx) {
	const uint32_t s = ra + k;
	if (s >= rb || m.nf == 0) return false;
	const uint32_t f = m.fidx[k];
	const uint2 fr = m.ftab[f];
	*idx = fr.x + (s - m.fstart[f]);
	*lv = frag_level(fr);
	return true;
}

__device__ __forceinline__ uint32_t block_end(const SlotSpace& sp, uint32_t r) {
	const uint32_t ra = r * kPrRange;
	return r == sp.nranges - 1 ? sp.total : min(sp.total, ra + kPrRange);
}

// ---------------------------------------------------------------------------
// Flattening the live in-adjacency
// ---------------------------------------------------------------------------

// blk_live[r] = live slots of block r.
__global__ void __launch_bounds__(kPrThreads)
flat_count(SlotSpace sp, uint32_t* blk_live) {
	__shared__ BlockMap m;
	__shared__ uint32_t red[kPrThreads / 32];
	const uint32_t tid = threadIdx.x, lane = tid & 31u, wid = tid >> 5;
	const uint32_t r = blockIdx.x, ra = r * kPrRange, rb = block_end(sp, r);
	map_block(sp, r, ra, rb, m);
	uint32_t c = 0;
#pragma unroll
	for (int u = 0; u < kPrPerThread; u++) {
		uint32_t lv, idx;
		if (block_slot(m, ra, rb, u * kPrThreads + tid, &lv, &idx))
			c += !slot_deleted(sp.in.lt, lv, idx);
	}
#pragma unroll
	for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
	if (lane == 0) red[wid] = c;
	__syncthreads();
	if (tid == 0) {
		uint32_t t = 0;
		for (int w = 0; w < kPrThreads / 32; w++) t += red[w];
		blk_live[r] = t;
	}
}

// Writes the live slots of block r to flat_ids[blk_base[r] ...] in slot
// order, and flat_off[e] for every entry e that starts in the block
// (flat_off has V + 1 entries; the last block also writes the trailing ones).
__global__ void __launch_bounds__(kPrThreads)
flat_write(SlotSpace sp, const uint32_t* blk_base, uint32_t* flat_ids, uint32_t* flat_off) {
	constexpr int kGroups = kPrPerThread * (kPrThreads / 32);
	__shared__ BlockMap m;
	__shared__ uint16_t rank[kPrRange];
	__shared__ uint32_t gpre[kGroups];
	const uint32_t tid = threadIdx.x, lane = tid & 31u, wid = tid >> 5;
	const uint32_t r = blockIdx.x, ra = r * kPrRange, rb = block_end(sp, r);
	map_block(sp, r, ra, rb, m);
	uint32_t id[kPrPerThread], mask[kPrPerThread];
#pragma unroll
	for (int u = 0; u < kPrPerThread; u++) {
		uint32_t lv = 0, idx = 0;
		bool live = block_slot(m, ra, rb, u * kPrThreads + tid, &lv, &idx);
		if (live) live = !slot_deleted(sp.in.lt, lv, idx);
		id[u] = live ? __ldg(sp.in.lt->ids[lv] + idx) : 0u;
		mask[u] = __ballot_sync(0xffffffffu, live);
	}
	// slot order is k = u * kPrThreads + wid * 32 + lane: group u * 4 + wid
	if (lane == 0) {
#pragma unroll
		for (int u = 0; u < kPrPerThread; u++) gpre[u * (kPrThreads / 32) + wid] = __popc(mask[u]);
	}
	__syncthreads();
	if (wid == 0) {
		const uint32_t c = lane < (uint32_t)kGroups ? gpre[lane] : 0u;
		uint32_t x = c;
#pragma unroll
		for (int o = 1; o < 32; o <<= 1) {
			const uint32_t t = __shfl_up_sync(0xffffffffu, x, o);
			if (lane >= (uint32_t)o) x += t;
		}
		if (lane < (uint32_t)kGroups) gpre[lane] = x - c;
	}
	__syncthreads();
	const uint32_t base = __ldg(blk_base + r);
	const uint32_t below = (1u << lane) - 1u;
#pragma unroll
	for (int u = 0; u < kPrPerThread; u++) {
		const uint32_t k = u * kPrThreads + tid;
		const uint32_t rk = gpre[u * (kPrThreads / 32) + wid] + __popc(mask[u] & below);
		rank[k] = (uint16_t)rk;
		if ((mask[u] >> lane) & 1u) flat_ids[base + rk] = id[u];
	}
	__syncthreads();
	const uint32_t V = (uint32_t)sp.in.V;
	const bool last = r == sp.nranges - 1;
	const uint32_t e_begin = __ldg(sp.range_lb + r);
	const uint32_t e_end = last ? V + 1 : __ldg(sp.range_lb + r + 1);
	const uint32_t next = __ldg(blk_base + r + 1);
	for (uint32_t e = e_begin + tid; e < e_end; e += kPrThreads) {
		const uint32_t p = __ldg(sp.pos + e);
		flat_off[e] = p < rb ? base + rank[p - ra] : next;
	}
}

__global__ void flat_flags(const uint32_t* flat_off, uint64_t V, uint32_t* flags) {
	const uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (v >= V) return;
	flags[v] = __ldg(flat_off + v + 1) > __ldg(flat_off + v);
}

__global__ void flat_rows(const uint32_t* flat_off, const uint32_t* kidx, uint64_t V,
		uint32_t* nz_rows, uint32_t* nz_off, uint32_t* heads) {
	const uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (v >= V) return;
	const uint32_t o = __ldg(flat_off + v);
	if (__ldg(flat_off + v + 1) == o) return;
	const uint32_t k = __ldg(kidx + v);
	nz_rows[k] = (uint32_t)v;
	nz_off[k] = o;
	atomicOr(heads + (o >> 5), 1u << (o & 31u));
}

constexpr int kFlatPerLane = 8;                         // consecutive edges per lane
constexpr uint32_t kFlatTile = 32u * kFlatPerLane;      // edges per warp
constexpr uint32_t kFlatTileWords = kFlatTile / 32u;    // head words per tile
constexpr int kFlatWarps = 8;                           // warps per CTA

// tile_seg[t] = number of rows beginning before edge t * kFlatTile.
__global__ void flat_tiles(const uint32_t* nz_off, uint32_t R, uint32_t ntiles,
		uint32_t* tile_seg) {
	const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= ntiles) return;
	const uint32_t x = t * kFlatTile;
	uint32_t lo = 0, hi = R;
	while (lo < hi) {
		const uint32_t mid = (lo + hi) >> 1;
		if (__ldg(nz_off + mid) < x) lo = mid + 1; else hi = mid;
	}
	tile_seg[t] = lo;
}

// ---------------------------------------------------------------------------
// Iterations over the flat array
// ---------------------------------------------------------------------------

struct FlatArgs {
	const uint32_t* ids;       // E
	const uint32_t* heads;     // ntiles * kFlatTileWords + 1 words
	const uint32_t* nz_rows;   // R
	const uint32_t* nz_off;    // R
	const uint32_t* tile_seg;  // ntiles
	uint32_t E, R, ntiles;
	const uint32_t* outdeg;
	const double* contrib;
	double* contrib_next;
	double* pr_out;            // written when non-null (last iteration)
	double base;               // (1 - d) / N
	double d;
	double* carry_first;       // per tile: the part of a row begun before it
	double* carry_last;        // per tile: the part of a row that runs past it
};

__device__ __forceinline__ void flat_finish(const FlatArgs& a, uint32_t k, double s) {
	const uint32_t v = __ldg(a.nz_rows + k);
	const double pr = __dadd_rn(a.base, __dmul_rn(a.d, s));
	const uint32_t dg = __ldg(a.outdeg + v);
	a.contrib_next[v] = dg ? pr / (double)dg : 0.0;
	if (a.pr_out) a.pr_out[v] = pr;
}

// One warp per tile of kFlatTile edges; lane j takes the kFlatPerLane
// consecutive edges e0 + 8j ... e0 + 8j + 7 (two 16-byte id loads) and the
// matching byte of the tile's head bits.  Each lane adds its values
// serially: the part before its first head (lead) continues the row open
// from the lanes to its left, rows that begin and end inside the lane are
// complete, and the part after its last head (tail) is open to the right.
// One segmented warp scan over (has head, tail or lead) gives every lane
// the open row's total so far.  Finished row sums are staged in shared
// memory and turned into ranks 32 at a time at the end of the tile.
__global__ void __launch_bounds__(kFlatWarps * 32)
pr_flat_step(FlatArgs a) {
	__shared__ double rowsum[kFlatWarps][kFlatTile];
	const uint32_t lane = threadIdx.x & 31u, wid = threadIdx.x >> 5;
	const uint32_t t = blockIdx.x * kFlatWarps + wid;
	if (t >= a.ntiles) return;                       // whole warps leave together
	double* rs = rowsum[wid];
	const uint32_t e0 = t * kFlatTile;
	const uint32_t eb = e0 + lane * kFlatPerLane;    // this lane's first edge
	const unsigned char* hbytes = reinterpret_cast<const unsigned char*>(a.heads);
	const uint32_t hb = __ldg(hbytes + (size_t)t * (kFlatTile / 8) + lane);
	const uint32_t hnext = __ldg(hbytes + (size_t)(t + 1) * (kFlatTile / 8)) & 1u;
	uint32_t id[kFlatPerLane];
	if (eb + kFlatPerLane <= a.E) {
		const uint4 p0 = __ldcs(reinterpret_cast<const uint4*>(a.ids + eb));
		const uint4 p1 = __ldcs(reinterpret_cast<const uint4*>(a.ids + eb) + 1);
		id[0] = p0.x; id[1] = p0.y; id[2] = p0.z; id[3] = p0.w;
		id[4] = p1.x; id[5] = p1.y; id[6] = p1.z; id[7] = p1.w;
	} else {
#pragma unroll
		for (int i = 0; i < kFlatPerLane; i++)
			id[i] = eb + i < a.E ? __ldcs(a.ids + eb + i) : kNoId;
	}
	double x[kFlatPerLane];
#pragma unroll
	for (int i = 0; i < kFlatPerLane; i++)
		x[i] = id[i] != kNoId ? __ldg(a.contrib + id[i]) : 0.0;

	// heads in the lanes to the left
	const uint32_t nh = __popc(hb);
	uint32_t before = nh;
#pragma unroll
	for (int o = 1; o < 32; o <<= 1) {
		const uint32_t q = __shfl_up_sync(0xffffffffu, before, o);
		if (lane >= (uint32_t)o) before += q;
	}
	const uint32_t H = __shfl_sync(0xffffffffu, before, 31);   // heads in the tile
	before -= nh;
	// serial pass over the lane's values
	double acc = 0.0, lead = 0.0;
	uint32_t seen = 0;
#pragma unroll
	for (int i = 0; i < kFlatPerLane; i++) {
		if ((hb >> i) & 1u) {
			if (seen == 0) lead = acc;
			else rs[before + seen - 1] = acc;      // a row inside the lane
			seen++;
			acc = 0.0;
		}
		acc += x[i];
	}
	if (seen == 0) lead = acc;
	// open row total at the end of each lane: scan of (has head, value)
	bool f = nh != 0;
	double v = f ? acc : lead;
#pragma unroll
	for (int o = 1; o < 32; o <<= 1) {
		const double pv = __shfl_up_sync(0xffffffffu, v, o);
		const bool pf = __shfl_up_sync(0xffffffffu, (uint32_t)f, o) != 0u;
		if (lane >= (uint32_t)o) {
			if (!f) v = pv + v;
			f = f || pf;
		}
	}
	// the open row from the left ends at this lane's first head
	double open_in = __shfl_up_sync(0xffffffffu, v, 1);
	if (lane == 0) open_in = 0.0;
	if (nh != 0) {
		const double s = open_in + lead;
		if (before == 0) a.carry_first[t] = s;   // began before the tile
		else rs[before - 1] = s;
	}
	// the row open at the end of the tile
	const double open_out = __shfl_sync(0xffffffffu, v, 31);
	const bool closes = (uint64_t)e0 + kFlatTile >= a.E || hnext;
	if (lane == 31u) {
		if (H == 0) a.carry_first[t] = open_out;
		else if (closes) rs[H - 1] = open_out;
		else a.carry_last[t] = open_out;
	}
	__syncwarp();
	const uint32_t done = (H > 0 && !closes) ? H - 1 : H;
	const uint32_t seg0 = __ldg(a.tile_seg + t);
	for (uint32_t r = lane; r < done; r += 32u) flat_finish(a, seg0 + r, rs[r]);
}

// Rows that cross tile boundaries: boundary t (edge t * kFlatTile) owns the
// row that crosses it if that row began in tile t - 1; its value is
// carry_last[t - 1] + carry_first[t] + ... + carry_first[t1], t1 the tile
// of its last edge.  A warp takes 32 boundaries; rows over more than four
// tiles are summed by the whole warp.
__global__ void pr_flat_fixup(FlatArgs a) {
	const uint32_t lane = threadIdx.x & 31u;
	const uint32_t w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	const uint32_t t = w * 32u + lane + 1u;
	bool own = false;
	uint32_t k = 0, t1 = 0;
	if (t < a.ntiles) {
		const uint32_t b = t * kFlatTile;
		const bool head = __ldg(a.heads + t * kFlatTileWords) & 1u;   // bit of edge b
		const uint32_t S = __ldg(a.tile_seg + t);
		if (!head && S > 0) {
			k = S - 1;
			const uint32_t start = __ldg(a.nz_off + k);
			if (start + kFlatTile >= b) {
				const uint32_t end = k + 1 < a.R ? __ldg(a.nz_off + k + 1) : a.E;
				t1 = (end - 1) / kFlatTile;
				own = true;
			}
		}
	}
	if (own && t1 - t < 4) {
		double s = __ldcg(a.carry_last + t - 1);
		for (uint32_t x = t; x <= t1; x++) s += __ldcg(a.carry_first + x);
		flat_finish(a, k, s);
		own = false;
	}
	uint32_t mm = __ballot_sync(0xffffffffu, own);
	while (mm) {
		const int src = __ffs(mm) - 1;
		mm &= mm - 1;
		const uint32_t tt = __shfl_sync(0xffffffffu, t, src);
		const uint32_t kk = __shfl_sync(0xffffffffu, k, src);
		const uint32_t tt1 = __shfl_sync(0xffffffffu, t1, src);
		double s = 0.0;
		for (uint32_t x = tt + lane; x <= tt1; x += 32u) s += __ldcg(a.carry_first + x);
#pragma unroll
		for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
		if (lane == 0) flat_finish(a, kk, __ldcg(a.carry_last + tt - 1) + s);
	}
}

// Vertices without in-edges: rank pr, contrib pr / out_degree.
__global__ void pr_empty_rows(const uint32_t* flat_off, const uint32_t* outdeg, uint64_t V,
		double pr, double* contrib, double* pr_out) {
	const uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (v >= V) return;
	if (__ldg(flat_off + v + 1) != __ldg(flat_off + v)) return;
	if (contrib) {
		const uint32_t dg = __ldg(outdeg + v);
		contrib[v] = dg ? pr / (double)dg : 0.0;
	}
	if (pr_out) pr_out[v] = pr;
}

// ---------------------------------------------------------------------------
// Fragment-walking iteration (no flat array)
// ---------------------------------------------------------------------------

struct PrArgs {
	SlotSpace sp;
	const uint32_t* outdeg;
	const double* contrib;
	double* contrib_next;
	double* pr_out;            // written when non-null (last iteration)
	double base;               // (1 - d) / N
	double d;
	double* carry_first;       // per block
	double* carry_last;        // per block
};

__device__ __forceinline__ void pr_finish(const PrArgs& a, uint32_t v, double s) {
	const double pr = __dadd_rn(a.base, __dmul_rn(a.d, s));
	const uint32_t dg = __ldg(a.outdeg + v);
	a.contrib_next[v] = dg ? pr / (double)dg : 0.0;
	if (a.pr_out) a.pr_out[v] = pr;
}

__device__ __forceinline__ void pr_emit(const PrArgs& a, uint32_t r, uint32_t ra, uint32_t rb,
		uint32_t e, uint32_t start, uint32_t end, double s) {
	if (start < ra) a.carry_first[r] = s;          // began before the block
	else if (end > rb) a.carry_last[r] = s;        // runs past its end
	else pr_finish(a, e, s);
}

// One CTA per block of kPrRange virtual slots.  Phase 1 streams the block's
// slots (slot ra + u * kPrThreads + tid for thread tid, coalesced id loads,
// all loads of a thread issued before any value is used) into shared
// memory; phase 2 sums each vertex's values (one thread per short vertex, a
// warp per long one).  A vertex straddling blocks leaves a partial per block
// that pr_fixup adds in block order.
__global__ void __launch_bounds__(kPrThreads)
pr_pull_step(PrArgs a) {
	__shared__ BlockMap m;
	__shared__ double vals[kPrRange];
	__shared__ uint32_t longs[kPrRange / kPrLong + 2];
	__shared__ uint32_t sh_nlong;
	const uint32_t tid = threadIdx.x, lane = tid & 31u, wid = tid >> 5;
	const uint32_t r = blockIdx.x, ra = r * kPrRange, rb = block_end(a.sp, r);
	if (tid == 0) sh_nlong = 0;
	map_block(a.sp, r, ra, rb, m);
	const uint32_t eb = m.eb, ee = m.ee;
	{
		const LevelTab* lt = a.sp.in.lt;
		uint32_t id[kPrPerThread], dw[kPrPerThread], bit[kPrPerThread];
		bool in[kPrPerThread];
#pragma unroll
		for (int u = 0; u < kPrPerThread; u++) {
			uint32_t lv = 0, idx = 0;
			in[u] = block_slot(m, ra, rb, u * kPrThreads + tid, &lv, &idx);
			id[u] = 0; dw[u] = 0; bit[u] = 0;
			if (in[u]) {
				id[u] = __ldg(lt->ids[lv] + idx);
				dw[u] = __ldg(lt->del[lv] + (idx >> 5));
				bit[u] = idx & 31u;
			}
		}
		double x[kPrPerThread];
#pragma unroll
		for (int u = 0; u < kPrPerThread; u++)
			x[u] = (in[u] && !((dw[u] >> bit[u]) & 1u)) ? __ldg(a.contrib + id[u]) : 0.0;
#pragma unroll
		for (int u = 0; u < kPrPerThread; u++) vals[u * kPrThreads + tid] = x[u];
	}
	__syncthreads();

	// phase 2: per-entry sums (short entries by one thread, in slot order)
	for (uint32_t e = eb + tid; e < ee; e += kPrThreads) {
		const uint32_t start = __ldg(a.sp.pos + e), end = __ldg(a.sp.pos + e + 1);
		const uint32_t s0 = max(start, ra), s1 = min(end, rb);
		if (s1 > s0 + kPrLong) {
			const uint32_t q = atomicAdd(&sh_nlong, 1u);
			longs[q] = e;
			continue;
		}
		double s = 0.0;
		for (uint32_t k = s0; k < s1; k++) s += vals[k - ra];
		pr_emit(a, r, ra, rb, e, start, end, s);
	}
	__syncthreads();
	// long entries: one warp each, fixed lane stride and tree order
	for (uint32_t q = wid; q < sh_nlong; q += kPrThreads / 32) {
		const uint32_t e = longs[q];
		const uint32_t start = __ldg(a.sp.pos + e), end = __ldg(a.sp.pos + e + 1);
		const uint32_t s0 = max(start, ra), s1 = min(end, rb);
		double s = 0.0;
		for (uint32_t k = s0 + lane; k < s1; k += 32) s += vals[k - ra];
#pragma unroll
		for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
		if (lane == 0) pr_emit(a, r, ra, rb, e, start, end, s);
	}
}

// Vertices straddling block boundaries: the thread of boundary q handles the
// vertex that starts in block q-1 and crosses q*kPrRange.
__global__ void pr_fixup(PrArgs a) {
	const uint64_t q = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x + 1;
	if (q >= a.sp.nranges) return;
	const uint32_t s = (uint32_t)q * kPrRange;
	// last entry e with pos[e] <= s (pos[0] = 0 <= s)
	uint32_t lo = 0, hi = (uint32_t)a.sp.in.V;
	while (lo < hi) {
		const uint32_t mid = (lo + hi + 1) >> 1;
		if (__ldg(a.sp.pos + mid) <= s) lo = mid; else hi = mid - 1;
	}
	const uint32_t e = lo;
	if (e >= a.sp.in.V) return;
	const uint32_t start = __ldg(a.sp.pos + e), end = __ldg(a.sp.pos + e + 1);
	if (!(start < s && start >= s - kPrRange && end > s)) return;
	const uint32_t r2 = (end - 1) / kPrRange;
	double t = __ldcg(a.carry_last + (q - 1));
	for (uint32_t x = (uint32_t)q; x <= r2; x++) t += __ldcg(a.carry_first + x);
	pr_finish(a, e, t);
}

__global__ void pr_init(const uint32_t* outdeg, uint64_t V, double pr0,
		double* contrib, double* pr_out) {
	uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (v >= V) return;
	uint32_t dg = outdeg[v];
	contrib[v] = dg ? pr0 / (double)dg : 0.0;
	if (pr_out) pr_out[v] = pr0;
}

static SlotSpace slot_space(const lg_snapshot* sn) {
	SlotSpace sp;
	sp.in = sn->view(1);
	sp.pos = sn->in.slot_off.as<uint32_t>();
	sp.range_lb = sn->in.range_lb.as<uint32_t>();
	sp.total = (uint32_t)sn->in.n_frag_slots;
	sp.nranges = (uint32_t)std::max<uint64_t>(1, (sp.total + kPrRange - 1) / kPrRange);
	return sp;
}

static lg_status check_args(lg_snapshot* sn, int iterations, double damping, double* ranks) {
	if (!sn || !ranks) return set_error(LG_EINVAL, "null argument");
	if (!(damping > 0.0 && damping < 1.0))
		return set_error(LG_EINVAL, "damping must be in (0, 1)");
	if (iterations < 0) return set_error(LG_EINVAL, "iterations must be >= 0");
	if (!sn->in.present)
		return set_error(LG_ESTATE, "pull PageRank needs the in-CSR (reverse edges)");
	return LG_OK;
}

} // namespace lg

using namespace lg;

extern "C" lg_status lg_pagerank_pull(lg_snapshot* sn, int iterations,
		double damping, double* ranks) {
	clear_error();
	LG_TRY(check_args(sn, iterations, damping, ranks));
	lg_store* s = sn->store;
	LG_CUDA(cudaSetDevice(s->device), "cudaSetDevice");
	cudaStream_t st = s->stream;
	const uint64_t V = sn->V;
	if (V == 0) return LG_OK;
	const double N = (double)V;
	const double pr0 = 1.0 / N;
	const double base = (1.0 - damping) / N;
	const SlotSpace sp = slot_space(sn);
	const unsigned B = 256;
	DevBuf* sc = s->scratch;
	const uint32_t* outdeg = sn->out.deg.as<uint32_t>();

	// flat in-adjacency of the snapshot
	LG_TRY(sc[7].reserve(2ull * (sp.nranges + 1) * sizeof(uint32_t)));
	uint32_t* blk_live = sc[7].as<uint32_t>();
	uint32_t* blk_base = blk_live + sp.nranges + 1;
	flat_count<<<sp.nranges, kPrThreads, 0, st>>>(sp, blk_live);
	LG_CUDA(cudaGetLastError(), "flat_count");
	uint64_t E = 0;
	LG_TRY(exclusive_scan_u32(blk_live, blk_base, sp.nranges, sc[8], st, &E));
	if (E > 0xffffffffull - 2 * kFlatTile)
		return set_error(LG_ENOTSUP, "more than 2^32 - %u live in-edges", 2 * kFlatTile);
	const uint32_t ntiles = (uint32_t)((E + kFlatTile - 1) / kFlatTile);
	LG_TRY(sc[3].reserve(std::max<uint64_t>(E, 1) * sizeof(uint32_t)));
	LG_TRY(sc[5].reserve(2 * (V + 1) * sizeof(uint32_t)));
	uint32_t* flat_off = sc[5].as<uint32_t>();
	uint32_t* kidx = flat_off + V + 1;
	flat_write<<<sp.nranges, kPrThreads, 0, st>>>(sp, blk_base, sc[3].as<uint32_t>(), flat_off);
	LG_CUDA(cudaGetLastError(), "flat_write");
	LG_TRY(sc[9].reserve(V * sizeof(uint32_t)));
	flat_flags<<<grid_for(V, B), B, 0, st>>>(flat_off, V, sc[9].as<uint32_t>());
	LG_CUDA(cudaGetLastError(), "flat_flags");
	uint64_t R = 0;
	LG_TRY(exclusive_scan_u32(sc[9].as<uint32_t>(), kidx, V, sc[8], st, &R));
	const uint64_t head_words = (uint64_t)ntiles * kFlatTileWords + 1;
	LG_TRY(sc[6].reserve((2 * std::max<uint64_t>(R, 1) + ntiles + head_words) * sizeof(uint32_t)));
	uint32_t* nz_rows = sc[6].as<uint32_t>();
	uint32_t* nz_off = nz_rows + std::max<uint64_t>(R, 1);
	uint32_t* tile_seg = nz_off + std::max<uint64_t>(R, 1);
	uint32_t* heads = tile_seg + ntiles;
	LG_CUDA(cudaMemsetAsync(heads, 0, head_words * sizeof(uint32_t), st), "clear heads");
	flat_rows<<<grid_for(V, B), B, 0, st>>>(flat_off, kidx, V, nz_rows, nz_off, heads);
	LG_CUDA(cudaGetLastError(), "flat_rows");
	if (ntiles > 0) {
		flat_tiles<<<grid_for(ntiles, B), B, 0, st>>>(nz_off, (uint32_t)R, ntiles, tile_seg);
		LG_CUDA(cudaGetLastError(), "flat_tiles");
	}
	s->launches += 2 + 3 + 1 + 3 + 1 + (ntiles > 0);

	FlatArgs a;
	a.ids = sc[3].as<uint32_t>();
	a.heads = heads;
	a.nz_rows = nz_rows;
	a.nz_off = nz_off;
	a.tile_seg = tile_seg;
	a.E = (uint32_t)E;
	a.R = (uint32_t)R;
	a.ntiles = ntiles;
	a.outdeg = outdeg;
	a.base = base;
	a.d = damping;
	LG_TRY(sc[0].reserve(V * sizeof(double)));
	LG_TRY(sc[1].reserve(V * sizeof(double)));
	LG_TRY(sc[2].reserve(2ull * std::max<uint32_t>(ntiles, 1) * sizeof(double)));
	a.carry_first = sc[2].as<double>();
	a.carry_last = a.carry_first + std::max<uint32_t>(ntiles, 1);
	const bool dev_out = is_device_pointer(ranks);
	double* pr_buf = ranks;
	if (!dev_out) {
		LG_TRY(sc[4].reserve(V * sizeof(double)));
		pr_buf = sc[4].as<double>();
	}
	double* c0 = sc[0].as<double>();
	double* c1 = sc[1].as<double>();
	pr_init<<<grid_for(V, B), B, 0, st>>>(outdeg, V, pr0, c0, iterations == 0 ? pr_buf : nullptr);
	pr_empty_rows<<<grid_for(V, B), B, 0, st>>>(flat_off, outdeg, V, base, c1, nullptr);
	LG_CUDA(cudaGetLastError(), "pr_init");
	s->launches += 2;
	const unsigned step_blocks = (ntiles + kFlatWarps - 1) / kFlatWarps;
	const unsigned fix_blocks = grid_for(ntiles, B);   // a thread per tile boundary
	for (int it = 0; it < iterations; it++) {
		a.contrib = (it & 1) ? c1 : c0;
		a.contrib_next = (it & 1) ? c0 : c1;
		a.pr_out = (it == iterations - 1) ? pr_buf : nullptr;
		if (ntiles > 0) {
			pr_flat_step<<<step_blocks, kFlatWarps * 32, 0, st>>>(a);
			s->launches++;
		}
		if (ntiles > 1) {
			pr_flat_fixup<<<fix_blocks, B, 0, st>>>(a);
			s->launches++;
		}
		if (it == 0 && iterations > 1) {
			// c0 still holds pr0 / out_degree for vertices without in-edges
			pr_empty_rows<<<grid_for(V, B), B, 0, st>>>(flat_off, outdeg, V, base, c0, nullptr);
			s->launches++;
		}
	}
	if (iterations > 0) {
		pr_empty_rows<<<grid_for(V, B), B, 0, st>>>(flat_off, outdeg, V, base, nullptr, pr_buf);
		s->launches++;
	}
	LG_CUDA(cudaGetLastError(), "pr_flat_step");
	if (!dev_out) {
		LG_TRY(copy_out(s, ranks, pr_buf, V * sizeof(double)));
		LG_CUDA(cudaStreamSynchronize(st), "pagerank");
	}
	return LG_OK;
}

// ---------------------------------------------------------------------------
// PageRank without device allocation.
//
// lg_pagerank_pull keeps its per-iteration vectors in store-owned scratch
// that it grows with cudaMalloc.  Some callers cannot have the library
// allocate: a thread that is capturing work into a CUDA graph (cudaMalloc
// and cudaFree are not allowed while its stream is being captured), or a
// process whose device memory is already handed out to another allocator,
// where a new cudaMalloc can fail or stall on a device-wide synchronisation.
// For them this variant runs the fragment-walking kernels on a fixed scratch
// area that is part of the library image: LG_NOALLOC_SCRATCH_BYTES of device
// memory, reserved on every GPU that loads the library, until the process
// exits.
// ---------------------------------------------------------------------------

namespace lg {

static __device__ __align__(256) unsigned char g_noalloc_scratch[LG_NOALLOC_SCRATCH_BYTES];

} // namespace lg

extern "C" lg_status lg_pagerank_pull_noalloc(lg_snapshot* sn, int iterations,
		double damping, double* ranks) {
	clear_error();
	LG_TRY(check_args(sn, iterations, damping, ranks));
	lg_store* s = sn->store;
	const uint64_t V = sn->V;
	const SlotSpace sp = slot_space(sn);
	const uint64_t nranges = sp.nranges;
	// contrib (two vectors), the result staged for host outputs, carries
	const uint64_t need = 3 * V * sizeof(double) + 2 * nranges * sizeof(double);
	if (need > LG_NOALLOC_SCRATCH_BYTES)
		return set_error(LG_EINVAL, "graph needs %llu scratch bytes, more than the %llu "
				"this entry point has (24 B per vertex + 16 B per %u in-CSR slots)",
				(unsigned long long)need, (unsigned long long)LG_NOALLOC_SCRATCH_BYTES,
				kPrRange);
	LG_CUDA(cudaSetDevice(s->device), "cudaSetDevice");
	// Device address of the scratch array, looked up once per device with
	// that device current (host code must not use the symbol itself).
	static std::mutex mu;
	static void* scratch_of[LG_NOALLOC_MAX_DEVICES] = {};
	if (s->device < 0 || s->device >= LG_NOALLOC_MAX_DEVICES)
		return set_error(LG_ENOTSUP, "device ordinal %d beyond %d", s->device,
				LG_NOALLOC_MAX_DEVICES);
	void* base = nullptr;
	{
		std::lock_guard<std::mutex> lk(mu);
		if (!scratch_of[s->device]) {
			void* p = nullptr;
			LG_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch), "cudaGetSymbolAddress");
			scratch_of[s->device] = p;
		}
		base = scratch_of[s->device];
	}
	cudaStream_t st = s->stream;
	double* c0 = (double*)base;
	double* c1 = c0 + V;
	double* staged = c1 + V;
	double* carries = staged + V;

	PrArgs a;
	a.sp = sp;
	a.outdeg = sn->out.deg.as<uint32_t>();
	a.base = (1.0 - damping) / (double)V;
	a.d = damping;
	a.carry_first = carries;
	a.carry_last = carries + nranges;
	const bool dev_out = is_device_pointer(ranks);
	double* pr_buf = dev_out ? ranks : staged;
	pr_init<<<grid_for(V, 256), 256, 0, st>>>(a.outdeg, V, 1.0 / (double)V, c0,
			iterations == 0 ? pr_buf : nullptr);
	for (int it = 0; it < iterations; it++) {
		a.contrib = (it & 1) ? c1 : c0;
		a.contrib_next = (it & 1) ? c0 : c1;
		a.pr_out = (it == iterations - 1) ? pr_buf : nullptr;
		pr_pull_step<<<nranges, kPrThreads, 0, st>>>(a);
		if (nranges > 1) pr_fixup<<<grid_for(nranges, 256), 256, 0, st>>>(a);
	}
	LG_CUDA(cudaGetLastError(), "pagerank noalloc");
	s->launches += 1 + (uint64_t)iterations * (nranges > 1 ? 2 : 1);
	if (!dev_out) {
		LG_CUDA(cudaMemcpyAsync(ranks, pr_buf, V * sizeof(double), cudaMemcpyDeviceToHost, st),
				"copy result");
		s->d2h_bytes += V * sizeof(double);
		LG_CUDA(cudaStreamSynchronize(st), "pagerank noalloc");
	}
	return LG_OK;
}
