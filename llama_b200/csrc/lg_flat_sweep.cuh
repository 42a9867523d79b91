// lg_flat_sweep.cuh - one pass of "row sum of gathered edge values" over a
// flat CSR (lg_flat.cuh), shared by PageRank (lg_pagerank.cu) and the
// weighted fixed-point solves of the adjoint PageRank (lg_adjoint.cu).
//
// flat_sweep_tile gives each warp a tile of kFlatTile consecutive edges, 8 per
// lane: it issues the tile's id loads and the op's value loads up front,
// adds each lane's values serially and joins the lanes with one segmented
// warp scan keyed by the head bits; a row that runs past a tile boundary
// leaves partials (carry_first, carry_last) that flat_sweep_fixup_body adds in
// tile order, so every row's sum is formed in a fixed order (deterministic).
// No block barriers: each warp stages its finished row sums in its own
// shared memory and hands them to the op 32 rows at a time.  Each user
// wraps the two bodies in kernels of its own name (pr_flat_step, ...), so
// launch lists and profiles name the computation.
//
// An Op supplies
//   bool   skip() const                      the whole launch is a no-op
//   void   values(eb, id[8], x[8]) const     the 8 edge values of a lane
//                                            (id = kNoId past the end)
//   double finish(k, s) const                row k (index into nz_rows) has
//                                            sum s; returns its residual term
//   void   residual(r) const                 one warp's residual total
//   static constexpr bool kResidual          finish() returns something
#ifndef LG_FLAT_SWEEP_CUH_
#define LG_FLAT_SWEEP_CUH_

#include "lg_flat.cuh"

namespace lg {

// Warps (tiles) per CTA of a tile kernel.  Small CTAs let a finished CTA's
// slots refill without waiting for its slowest tile: 4 warps measured 1.6 %
// faster than 8 and 4.5 % faster than 16 on a PageRank iteration over a
// 256 M-edge in-CSR.
constexpr int kFlatWarps = 4;
// Warps per CTA of the persistent loop kernels, whose CTAs stay resident.
constexpr int kFlatLoopWarps = 8;

struct FlatTiles {
	const uint32_t* ids;       // E
	const uint32_t* heads;     // ntiles * kFlatTileWords + 1 words
	const uint32_t* nz_off;    // R
	const uint32_t* tile_seg;  // ntiles
	uint32_t E, R, ntiles;
	double* carry_first;       // per tile: the part of a row begun before it
	double* carry_last;        // per tile: the part of a row that runs past it
};

inline FlatTiles flat_tiles(const FlatCsr& f, double* carries) {
	FlatTiles t;
	t.ids = f.ids.as<uint32_t>();
	t.heads = f.heads();
	t.nz_off = f.nz_off();
	t.tile_seg = f.tile_seg();
	t.E = (uint32_t)f.E;
	t.R = (uint32_t)f.R;
	t.ntiles = f.ntiles;
	t.carry_first = carries;
	t.carry_last = carries + (f.ntiles > 0 ? f.ntiles : 1);
	return t;
}

// Lane j of the warp owning tile t takes edges e0 + 8j ... e0 + 8j + 7 and
// the matching byte of the tile's head bits.  Each lane adds its values
// serially: the part before its first head (lead) continues the row open
// from the lanes to its left, rows that begin and end inside the lane are
// complete, and the part after its last head (tail) is open to the right.
// One segmented warp scan over (has head, tail or lead) gives every lane the
// open row's total so far.
//
// Processes tile t with the calling warp (rs: the warp's kFlatTile doubles
// of shared memory) and returns the lane's residual terms.
template <class Op>
__device__ __forceinline__ double flat_sweep_one(const FlatTiles& a, const Op& op, double* rs,
		uint32_t t) {
	const uint32_t lane = threadIdx.x & 31u;
	const uint32_t e0 = t * kFlatTile;
	const uint32_t eb = e0 + lane * kFlatPerLane;    // this lane's first edge
	const unsigned char* hbytes = reinterpret_cast<const unsigned char*>(a.heads);
	const uint32_t hb = __ldg(hbytes + (size_t)t * (kFlatTile / 8) + lane);
	const uint32_t hnext = __ldg(hbytes + (size_t)(t + 1) * (kFlatTile / 8)) & 1u;
	uint32_t id[kFlatPerLane];
	if (eb + kFlatPerLane <= a.E) {
		// one 32-byte load per lane (eb is a multiple of 8), evict-first so
		// the streamed ids do not push the gathered values out of L2
		asm("ld.global.cs.v8.u32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
			: "=r"(id[0]), "=r"(id[1]), "=r"(id[2]), "=r"(id[3]),
			  "=r"(id[4]), "=r"(id[5]), "=r"(id[6]), "=r"(id[7])
			: "l"(a.ids + eb));
	} else {
#pragma unroll
		for (int i = 0; i < kFlatPerLane; i++)
			id[i] = eb + i < a.E ? __ldcs(a.ids + eb + i) : kNoId;
	}
	double x[kFlatPerLane];
	op.values(eb, id, x);

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
	// Open row total at the end of each lane: a segmented scan in which a
	// lane adds the value o lanes to its left while that lane is still in
	// its open row, i.e. at or right of `start`, the nearest lane at or left
	// of it with a head (-1: none).  The segment bounds come from one ballot,
	// so each step moves only the value (two shuffles, each a slot of the L1
	// data pipe that the gathers keep busy), not a flag beside it.
	const uint32_t hm = __ballot_sync(0xffffffffu, nh != 0);
	const uint32_t with_head = hm & ((2u << lane) - 1u);
	const int start = with_head ? 31 - __clz(with_head) : -1;
	double v = nh != 0 ? acc : lead;
#pragma unroll
	for (int o = 1; o < 32; o <<= 1) {
		const double pv = __shfl_up_sync(0xffffffffu, v, o);
		if (lane >= (uint32_t)o && (int)lane - o >= start) v = pv + v;
	}
	// the open row from the left ends at this lane's first head
	double open_in = __shfl_up_sync(0xffffffffu, v, 1);
	if (lane == 0) open_in = 0.0;
	if (nh != 0) {
		const double s = open_in + lead;
		if (before == 0) a.carry_first[t] = s;   // began before the tile
		else rs[before - 1] = s;
	}
	// the row open at the end of the tile: lane 31's total
	const bool closes = (uint64_t)e0 + kFlatTile >= a.E || hnext;
	if (lane == 31u) {
		if (H == 0) a.carry_first[t] = v;
		else if (closes) rs[H - 1] = v;
		else a.carry_last[t] = v;
	}
	__syncwarp();
	const uint32_t done = (H > 0 && !closes) ? H - 1 : H;
	const uint32_t seg0 = __ldg(a.tile_seg + t);
	double res = 0.0;
	for (uint32_t r = lane; r < done; r += 32u) res += op.finish(seg0 + r, rs[r]);
	return res;
}

template <class Op>
__device__ __forceinline__ void flat_sweep_residual(const Op& op, double res) {
	if (Op::kResidual) {
#pragma unroll
		for (int o = 16; o > 0; o >>= 1) res += __shfl_xor_sync(0xffffffffu, res, o);
		if ((threadIdx.x & 31u) == 0 && res != 0.0) op.residual(res);
	}
}

// Body of a kernel launched with kFlatWarps * 32 threads per CTA and one
// CTA per kFlatWarps tiles: warp w of CTA b takes tile b * kFlatWarps + w.
// rowsum is the CTA's shared double[kFlatWarps][kFlatTile].
template <class Op>
__device__ __forceinline__ void flat_sweep_tile(const FlatTiles& a, const Op& op,
		double (*rowsum)[kFlatTile]) {
	const uint32_t wid = threadIdx.x >> 5;
	const uint32_t t = blockIdx.x * kFlatWarps + wid;
	if (t >= a.ntiles || op.skip()) return;          // whole warps leave together
	flat_sweep_residual(op, flat_sweep_one(a, op, rowsum[wid], t));
}

// The persistent form: a grid of a few CTAs per SM whose warps loop over the
// tiles (warp w of CTA b: tiles b * kFlatLoopWarps + w, then every gridDim.x *
// kFlatLoopWarps further), so no warp slot idles while a CTA waits for its
// slowest warp.  rowsum is the CTA's shared double[kFlatLoopWarps][kFlatTile].
template <class Op>
__device__ __forceinline__ void flat_sweep_loop(const FlatTiles& a, const Op& op,
		double (*rowsum)[kFlatTile]) {
	if (op.skip()) return;
	const uint32_t wid = threadIdx.x >> 5;
	const uint32_t stride = gridDim.x * kFlatLoopWarps;
	double res = 0.0;
	for (uint32_t t = blockIdx.x * kFlatLoopWarps + wid; t < a.ntiles; t += stride) {
		res += flat_sweep_one(a, op, rowsum[wid], t);
		__syncwarp();                     // rowsum is reused by the next tile
	}
	flat_sweep_residual(op, res);
}

// Rows that cross tile boundaries: boundary t (edge t * kFlatTile) owns the
// row that crosses it if that row began in tile t - 1; its value is
// carry_last[t - 1] + carry_first[t] + ... + carry_first[t1], t1 the tile
// of its last edge.  A warp takes 32 boundaries; rows over more than four
// tiles are summed by the whole warp.
template <class Op>
__device__ __forceinline__ void flat_sweep_fixup_body(const FlatTiles& a, const Op& op) {
	if (op.skip()) return;
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
	double res = 0.0;
	if (own && t1 - t < 4) {
		double s = __ldcg(a.carry_last + t - 1);
		for (uint32_t x = t; x <= t1; x++) s += __ldcg(a.carry_first + x);
		res += op.finish(k, s);
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
		if (lane == 0) res += op.finish(kk, __ldcg(a.carry_last + tt - 1) + s);
	}
	if (Op::kResidual) {
#pragma unroll
		for (int o = 16; o > 0; o >>= 1) res += __shfl_xor_sync(0xffffffffu, res, o);
		if (lane == 0 && res != 0.0) op.residual(res);
	}
}

// Launch shapes: a CTA of kFlatWarps warps per kFlatWarps tiles; a thread
// per tile boundary for the fix-up (kFixupThreads per CTA).
inline unsigned flat_sweep_blocks(uint32_t ntiles) {
	return (ntiles + kFlatWarps - 1) / kFlatWarps;
}
// Persistent grid: ctas_per_sm CTAs on each of sms SMs, never more CTAs
// than tiles need.
inline unsigned flat_loop_blocks(uint32_t ntiles, int sms, int ctas_per_sm) {
	const uint64_t g = (uint64_t)sms * (uint64_t)ctas_per_sm;
	const unsigned need = (ntiles + kFlatLoopWarps - 1) / kFlatLoopWarps;
	return (unsigned)(g < need ? g : need);
}
constexpr unsigned kFixupThreads = 256;

// A sweep launcher: the tile kernel (one CTA per kFlatWarps tiles) when
// ctas_per_sm is 0, else the persistent loop kernel whose register cap
// allows that many resident CTAs (4, 6 or 8), on that many CTAs per SM.
template <class Op, class TileK, class LoopK4, class LoopK6, class LoopK8>
inline void launch_flat_sweep(const FlatTiles& a, const Op& op, int sms, int ctas_per_sm,
		cudaStream_t st, TileK tile_k, LoopK4 loop4, LoopK6 loop6, LoopK8 loop8) {
	if (a.ntiles == 0) return;
	if (ctas_per_sm <= 0) {
		tile_k<<<flat_sweep_blocks(a.ntiles), kFlatWarps * 32, 0, st>>>(a, op);
		return;
	}
	const unsigned g = flat_loop_blocks(a.ntiles, sms, ctas_per_sm);
	if (ctas_per_sm <= 4) loop4<<<g, kFlatLoopWarps * 32, 0, st>>>(a, op);
	else if (ctas_per_sm <= 6) loop6<<<g, kFlatLoopWarps * 32, 0, st>>>(a, op);
	else loop8<<<g, kFlatLoopWarps * 32, 0, st>>>(a, op);
}
inline unsigned flat_fixup_blocks(uint32_t ntiles) { return grid_for(ntiles, kFixupThreads); }

} // namespace lg

#endif // LG_FLAT_SWEEP_CUH_
