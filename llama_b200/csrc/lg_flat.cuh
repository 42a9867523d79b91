// lg_flat.cuh - the virtual slot space of a snapshot direction cut into
// fixed blocks, and the flat single-level CSR built from it.
//
// The virtual slot space of a direction lists, in vertex order, the slots of
// every vertex's fragments newest first (slot_off is its prefix).  A block of
// kMapRange consecutive virtual slots maps its slots back to (level, index)
// through a shared-memory table of the fragments that touch it (BlockMap).
//
// A FlatCsr is that slot space with deleted slots removed: the live
// adjacency of the snapshot in iteration order, as one CSR
// (benchmark/tools/flatten.h merges the levels of a LLAMA graph into one
// level the same way, on the host).  Besides offsets and ids it carries
//   heads      bit per edge, set where a vertex's edges begin
//   nz_rows    R x u32, the vertices with edges, in order
//   nz_off     R x u32, where each of them begins
//   tile_seg   per kFlatTile edges, the rows begun before the tile
// for the tile kernels, and optionally a one-fragment-per-vertex view
// (frag_off = row index prefix, frags = {nz_off, len << 6 | level 0}, an
// all-zero deletion bitset) so the fragment-walking kernels run on it
// unchanged.
#ifndef LG_FLAT_CUH_
#define LG_FLAT_CUH_

#include "lg_device.cuh"

namespace lg {

constexpr int kMapThreads = 128;
constexpr int kMapPerThread = 8;
constexpr uint32_t kMapRange = kMapThreads * kMapPerThread;       // 1024 slots
static_assert(kMapRange == kBlockSlots, "range_lb is computed for kBlockSlots");
constexpr uint32_t kMapMaxFrags = kMapRange + 2 * LG_MAX_LEVELS;   // fragments touching a block

constexpr int kFlatPerLane = 8;                         // consecutive edges per lane
constexpr uint32_t kFlatTile = 32u * kFlatPerLane;      // edges per warp tile
constexpr uint32_t kFlatTileWords = kFlatTile / 32u;    // head words per tile

// One direction's virtual slot space cut into kMapRange-slot blocks.
struct SlotSpace {
	SnapCsr g;
	const uint32_t* pos;       // V + 1 virtual slot prefix
	const uint32_t* range_lb;  // nranges + 1 block entry bounds
	uint32_t total;            // pos[V]
	uint32_t nranges;
};

// Shared-memory map from the slots of one block to their fragments.
struct BlockMap {
	uint2 ftab[kMapMaxFrags];           // fragments of the block's entries
	uint32_t fstart[kMapMaxFrags + 1];  // their absolute virtual starts
	uint32_t fidx[kMapRange];           // block slot -> index into ftab
	uint32_t wsum[kMapThreads / 32];
	uint32_t eb, ee, nf;                // block entries [eb, ee), fragments
};

__device__ __forceinline__ uint32_t block_end(const SlotSpace& sp, uint32_t r) {
	const uint32_t ra = r * kMapRange;
	return r == sp.nranges - 1 ? sp.total : min(sp.total, ra + kMapRange);
}

// Builds m for block r (virtual slots [ra, rb)); all kMapThreads threads of
// the block call it, and it returns synchronised.
__device__ inline void map_block(const SlotSpace& sp, uint32_t r, uint32_t ra, uint32_t rb,
		BlockMap& m) {
	const uint32_t tid = threadIdx.x, lane = tid & 31u, wid = tid >> 5;
	const bool last_range = r == sp.nranges - 1;
	const uint32_t V = (uint32_t)sp.g.V;
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
	const uint32_t f_begin = __ldg(sp.g.frag_off + eb);
	uint32_t nf = (ee > eb) ? __ldg(sp.g.frag_off + ee) - f_begin : 0;
	// every fragment of an entry inside the block has a slot in the block,
	// and only the two end entries add others, so nf <= kMapMaxFrags
	if (nf > kMapMaxFrags) nf = kMapMaxFrags;
	const uint32_t vbase = __ldg(sp.pos + eb);
	uint32_t carry = 0;
	for (uint32_t c0 = 0; c0 < nf; c0 += kMapThreads) {
		const uint32_t i = c0 + tid;
		uint32_t len = 0;
		if (i < nf) { const uint2 fr = sp.g.frags[f_begin + i]; m.ftab[i] = fr; len = frag_len(fr); }
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
		for (uint32_t w2 = 0; w2 < kMapThreads / 32; w2++) tot += m.wsum[w2];
		carry += tot;
		__syncthreads();
	}
	if (tid == 0) { m.fstart[nf] = vbase + carry; m.nf = nf; }
	// slot -> fragment map: each fragment marks the first block slot it
	// covers (the last of the fragments starting at or before ra marks slot
	// 0), then an inclusive max-scan over the block's slots spreads the marks
	for (uint32_t k = tid; k < kMapRange; k += kMapThreads) m.fidx[k] = 0;
	__syncthreads();
	for (uint32_t i = tid; i < nf; i += kMapThreads) {
		const uint32_t st = m.fstart[i];
		if (st < rb) atomicMax(&m.fidx[st > ra ? st - ra : 0], i);
	}
	__syncthreads();
	{
		// thread t scans slots [8t, 8t + 8) serially, then a block scan of
		// the thread maxima carries the mark across threads
		uint32_t mx = 0, loc[kMapPerThread];
#pragma unroll
		for (int u = 0; u < kMapPerThread; u++) {
			mx = max(mx, m.fidx[tid * kMapPerThread + u]);
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
		for (int u = 0; u < kMapPerThread; u++)
			m.fidx[tid * kMapPerThread + u] = max(before, loc[u]);
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

// Slot space of direction dir (0 out, 1 in) of sn.
SlotSpace slot_space(const lg_snapshot* sn, int dir);

struct FlatCsr {
	uint64_t V = 0, E = 0, R = 0;
	uint32_t ntiles = 0;
	bool weighted = false;     // w holds the edge weights
	bool has_view = false;     // vfrags / vdel / vlt are built
	DevBuf off;                // V + 1 u32: row starts
	DevBuf kidx;               // V + 1 u32: rows with edges before each vertex
	DevBuf ids;                // E u32
	DevBuf w;                  // E u32 (weighted)
	DevBuf rows;               // nz_rows[R] nz_off[R] tile_seg[ntiles] heads[ntiles*8+1]
	DevBuf flags, scan_tmp, err;        // build scratch
	DevBuf vfrags, vdel, vlt;  // one-fragment-per-vertex view
	DevBuf nz_outdeg;          // R u32: out-degree of each row (PageRank, built on use)
	bool has_nz_outdeg = false;
	uint64_t rcap() const { return R > 0 ? R : 1; }
	const uint32_t* nz_rows() const { return rows.as<uint32_t>(); }
	const uint32_t* nz_off() const { return rows.as<uint32_t>() + rcap(); }
	const uint32_t* tile_seg() const { return rows.as<uint32_t>() + 2 * rcap(); }
	const uint32_t* heads() const { return rows.as<uint32_t>() + 2 * rcap() + ntiles; }
	// fragment view for the fragment-walking kernels (has_view); deg is the
	// snapshot's degree array of the same direction
	SnapCsr view(const uint32_t* deg) const {
		SnapCsr s;
		s.frag_off = kidx.as<uint32_t>();
		s.frags = vfrags.as<uint2>();
		s.lt = vlt.as<LevelTab>();
		s.deg = deg;
		s.V = V;
		return s;
	}
};

// Builds f from direction dir of sn on the store's stream, with the edge
// weights when every level that holds fragment slots has them, and the
// fragment view when `view`.  f's buffers are reused (grown) across builds.
lg_status build_flat(lg_snapshot* sn, int dir, FlatCsr& f, bool view);

} // namespace lg

// Hands a snapshot's flat CSR back to its store, which keeps up to two (their
// device memory) for the next lg_snapshot_flatten; the caller has synchronised
// the store's stream.  f may be null.
void lg_flat_release(lg_store* s, lg::FlatCsr* f);

#endif // LG_FLAT_CUH_
