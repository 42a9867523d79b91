// lg_msbfs.cu - BFS levels from many roots at once.
//
// Reference: the same task as lg_bfs (u_sssp_bfs / ll_b_sssp_unweighted_bfs,
// benchmark/benchmarks/sssp.h:219-300), run for every root: dist[root] = 0,
// level-synchronous, unreached vertices keep INT_MAX - 1.  The benchmark
// runs one BFS per root; since BFS levels are unique, the roots can share
// their traversals: every vertex carries a 64-bit mask per pass, one bit per
// root (bit-parallel multi-source BFS), so one edge visit serves up to 64
// BFSs whose frontiers cross it in the same step.
//
//   seen[v]   roots that reached v
//   cur[v]    roots whose frontier holds v at the current depth
//   nxt[v]    roots that reach v at the next depth (candidates)
//
// A step is top-down over the union frontier queue (out-CSR, balanced
// 1024-slot ranges: nxt[w] |= cur[u] & ~seen[w]) or bottom-up (every vertex
// some root has not reached ORs cur[] over its in-neighbours until every
// missing root is found; flat in-CSR when the snapshot has one).  A commit
// pass turns nxt into the new frontier, sets seen, and writes depth + 1 into
// the level arrays of the new roots' bits.
//
// lg_bc_batched runs Brandes' betweenness centrality on the same machinery,
// 64 sources per pass (see the section below).
#include "lg_expand.cuh"
#include "lg_flat.cuh"
#include "lg_tune.h"

namespace lg {

typedef unsigned long long u64;
constexpr int32_t kMsUnreached = LG_UNREACHED;
constexpr int kMsThreads = 256;
constexpr uint32_t kMsRange = 1024;     // largest slot range per warp

// Slots per warp range for a list of `total` slots over `nwarps` warps: the
// even share rounded up to 32, between 32 and kMsRange, so a small frontier
// is spread over many warps instead of a few long ones.
__device__ __forceinline__ uint32_t ms_range(uint32_t total, uint32_t nwarps) {
	uint32_t r = (uint32_t)(((uint64_t)total + nwarps - 1) / nwarps);
	r = (r + 31u) & ~31u;
	return min(max(r, 32u), kMsRange);
}
constexpr int kMsChunk = 8;            // in-neighbours per bottom-up round
constexpr int kMsMaxRoots = 64;        // roots per pass

__global__ void ms_fill(int32_t* levels, uint64_t n) {
	for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
			i += (uint64_t)gridDim.x * blockDim.x)
		levels[i] = kMsUnreached;
}

// Roots k of this pass: bit k of seen and cur, level 0, the root queue.
// ctr[0] queue length, ctr[1] out-degree sum of the queued roots.
__global__ void ms_roots(const int64_t* roots, int n, uint64_t V, const uint32_t* outdeg,
		u64* seen, u64* cur, int32_t* levels, uint32_t* queue, unsigned long long* ctr) {
	const int k = threadIdx.x;
	if (k >= n) return;
	const uint32_t v = (uint32_t)roots[k];
	atomicOr(seen + v, 1ull << k);
	const u64 old = atomicOr(cur + v, 1ull << k);
	levels[(uint64_t)k * V + v] = 0;
	// the first root to mark v queues it (duplicates share the entry)
	if (old == 0) {
		queue[atomicAdd(ctr, 1ull)] = v;
		atomicAdd(ctr + 1, (unsigned long long)__ldg(outdeg + v));
	}
}

__device__ __forceinline__ void ms_push(bool take, uint32_t item, uint32_t* queue,
		unsigned long long* len) {
	const unsigned m = __ballot_sync(0xffffffffu, take);
	if (!m) return;
	const uint32_t lane = threadIdx.x & 31u;
	const int leader = __ffs(m) - 1;
	unsigned long long base = 0;
	if ((int)lane == leader) base = atomicAdd(len, (unsigned long long)__popc(m));
	base = __shfl_sync(0xffffffffu, base, leader);
	if (take) queue[base + __popc(m & ((1u << lane) - 1u))] = item;
}

// Top-down: queue = union frontier, pos its slot prefix (pos[qlen] total);
// a candidate w goes to `cand` the first time its nxt turns non-zero.
__global__ void __launch_bounds__(kMsThreads)
ms_top_down(SnapCsr out, const uint32_t* queue, const uint32_t* pos, uint32_t qlen,
		const u64* cur, const u64* seen, u64* nxt, uint32_t* cand, unsigned long long* ncand) {
	const uint32_t total = __ldg(pos + qlen);
	const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
	const uint32_t range = ms_range(total, nwarps);
	const uint32_t nranges = (total + range - 1) / range;
	for (uint32_t r = warp; r < nranges; r += nwarps) {
		range_for_each(out, queue, pos, qlen, total, nranges, range, r,
			[&](bool act, uint32_t, uint32_t ov, uint32_t nbr, uint32_t, uint32_t) {
				bool first = false;
				if (act) {
					const u64 bits = __ldg(cur + ov) & ~__ldcg(seen + nbr);
					if (bits && (__ldcg(nxt + nbr) & bits) != bits)
						first = atomicOr(nxt + nbr, bits) == 0;
				}
				ms_push(first, nbr, cand, ncand);
			});
	}
}

// Bottom-up over a flat in-CSR: a thread takes kMsVerts vertices (blockDim
// apart) and ORs cur[] over kMsChunk in-neighbours of each per round until
// every root that has not reached the vertex is found, or the list ends.
// Vertices with more than `heavy` in-edges (LG_TUNE_MS_HEAVY, 512 by
// default) are left to ms_bottom_up_heavy, so no thread walks a hub's list
// alone.  One vertex and eight neighbours
// per round measured best at R-MAT scale 24 (16-root BFS 3.56 ms, against
// 3.66 for two vertices x 4, 3.93 for four x 4 and for two x 8).
constexpr int kMsVerts = 1;
__global__ void __launch_bounds__(kMsThreads)
ms_bottom_up_flat(const uint32_t* off, const uint32_t* ids, uint32_t V, u64 lanes,
		const u64* cur, const u64* seen, u64* nxt, uint32_t heavy) {
	const uint32_t base = blockIdx.x * (uint32_t)(kMsThreads * kMsVerts) + threadIdx.x;
	uint32_t k[kMsVerts], end[kMsVerts];
	u64 need[kMsVerts], got[kMsVerts];
#pragma unroll
	for (int j = 0; j < kMsVerts; j++) {
		const uint32_t v = base + j * kMsThreads;
		k[j] = 0; end[j] = 0; need[j] = 0; got[j] = 0;
		if (v < V) {
			need[j] = lanes & ~seen[v];
			if (need[j]) {
				k[j] = __ldg(off + v);
				end[j] = __ldg(off + v + 1);
				if (end[j] - k[j] > heavy) { end[j] = k[j]; need[j] = 0; }
			}
		}
	}
	bool more = true;
	while (more) {
		uint32_t u[kMsVerts][kMsChunk];
#pragma unroll
		for (int j = 0; j < kMsVerts; j++)
#pragma unroll
			for (int c = 0; c < kMsChunk; c++)
				u[j][c] = k[j] + c < end[j] ? __ldg(ids + k[j] + c) : kNoId;
		u64 f[kMsVerts][kMsChunk];
#pragma unroll
		for (int j = 0; j < kMsVerts; j++)
#pragma unroll
			for (int c = 0; c < kMsChunk; c++)
				f[j][c] = u[j][c] != kNoId ? __ldg(cur + u[j][c]) : 0ull;
		more = false;
#pragma unroll
		for (int j = 0; j < kMsVerts; j++) {
#pragma unroll
			for (int c = 0; c < kMsChunk; c++) got[j] |= f[j][c];
			if ((got[j] & need[j]) == need[j]) k[j] = end[j];
			else k[j] = min(k[j] + kMsChunk, end[j]);
			more |= k[j] < end[j];
		}
	}
#pragma unroll
	for (int j = 0; j < kMsVerts; j++) {
		const uint32_t v = base + j * kMsThreads;
		const u64 b = got[j] & need[j];
		if (b) nxt[v] = b;
	}
}

// Vertices of a flat in-CSR with more than `heavy` in-edges.
__global__ void ms_heavy_list(const uint32_t* off, uint32_t V, uint32_t* list,
		unsigned long long* n, uint32_t heavy) {
	const uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	const bool h = v < V && __ldg(off + v + 1) - __ldg(off + v) > heavy;
	ms_push(h, (uint32_t)v, list, n);
}

// Bottom-up for the heavy vertices (*nheavy of them in `list`): a warp per
// vertex ORs the frontier masks of 32 in-neighbours at a time until every
// root that has not reached the vertex is found, or the list ends.
__global__ void __launch_bounds__(kMsThreads)
ms_bottom_up_heavy(const uint32_t* off, const uint32_t* ids, const uint32_t* list,
		const unsigned long long* nheavy, u64 lanes, const u64* cur, const u64* seen, u64* nxt) {
	const uint32_t lane = threadIdx.x & 31u;
	const uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
	const uint64_t n = *nheavy;
	for (uint64_t i = warp; i < n; i += nwarps) {
		const uint32_t v = __ldg(list + i);
		const u64 need = lanes & ~seen[v];
		if (!need) continue;
		const uint32_t k1 = __ldg(off + v + 1);
		u64 got = 0;
		for (uint32_t b = __ldg(off + v); b < k1; b += 32u * kMsChunk) {
			u64 f = 0;
#pragma unroll
			for (int c = 0; c < kMsChunk; c++) {
				const uint32_t k = b + c * 32u + lane;
				if (k < k1) f |= __ldg(cur + __ldg(ids + k));
			}
			got |= ((u64)__reduce_or_sync(0xffffffffu, (uint32_t)(f >> 32)) << 32)
				| __reduce_or_sync(0xffffffffu, (uint32_t)f);
			if ((got & need) == need) break;
		}
		if (lane == 0 && (got & need)) nxt[v] = got & need;
	}
}

// Bottom-up over the snapshot's fragments (no flat in-CSR): a thread per
// vertex walks its fragments, skipping deleted slots.
__global__ void __launch_bounds__(kMsThreads)
ms_bottom_up(SnapCsr in, u64 lanes, const u64* cur, const u64* seen, u64* nxt) {
	const uint64_t v64 = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (v64 >= in.V) return;
	const uint32_t v = (uint32_t)v64;
	const u64 need = lanes & ~seen[v];
	if (!need) return;
	u64 got = 0;
	const uint32_t f0 = __ldg(in.frag_off + v), f1 = __ldg(in.frag_off + v + 1);
	for (uint32_t f = f0; f < f1 && (got & need) != need; f++) {
		const uint2 fr = in.frags[f];
		const uint32_t lv = frag_level(fr), n = frag_len(fr);
		const uint32_t* ids = in.lt->ids[lv] + fr.x;
		for (uint32_t k = 0; k < n && (got & need) != need; k++) {
			if (slot_deleted(in.lt, lv, fr.x + k)) continue;
			got |= __ldg(cur + __ldg(ids + k));
		}
	}
	if (got & need) nxt[v] = got & need;
}

// Commit candidates (list, or every vertex when list is null): new roots'
// bits become the next frontier (cur2, zero before), are added to seen and
// get level depth + 1; the vertex joins the next queue.  ctr[0] next queue
// length, ctr[1] its out-degree sum, ctr[2] OR of the new bits.
//
// A CTA takes kCommitPer rounds of kMsThreads consecutive entries.  The
// level rows are written root by root for all threads of a warp alike, so
// the lanes holding bit k write row k at consecutive vertices together.
// The queue slots and the counters are taken once per CTA (a dense step
// commits every vertex, and one atomic per warp on the same three counters
// serialised in L2).
constexpr int kCommitPer = 4;
__global__ void __launch_bounds__(kMsThreads)
ms_commit(const uint32_t* list, uint32_t n, uint32_t depth1, uint64_t V,
		int nroots, u64* nxt, u64* seen, u64* cur2, int32_t* levels, const uint32_t* outdeg,
		uint32_t* queue, unsigned long long* ctr) {
	constexpr int kWarps = kMsThreads / 32;
	__shared__ uint32_t s_cnt[kWarps];
	__shared__ unsigned long long s_e[kWarps];
	__shared__ u64 s_any[kWarps];
	__shared__ unsigned long long s_base;
	const uint32_t lane = threadIdx.x & 31u, wid = threadIdx.x >> 5;
	const uint64_t b0 = (uint64_t)blockIdx.x * (kMsThreads * kCommitPer) + threadIdx.x;
	uint32_t ws[kCommitPer];
	unsigned masks[kCommitPer];
	uint32_t cnt = 0;
	unsigned long long e = 0;
	u64 any = 0;
#pragma unroll
	for (int r = 0; r < kCommitPer; r++) {
		const uint64_t i = b0 + (uint64_t)r * kMsThreads;
		uint32_t w = 0;
		u64 bits = 0;
		if (i < n) {
			w = list ? __ldg(list + i) : (uint32_t)i;
			const u64 c = nxt[w];
			if (c) {
				nxt[w] = 0;
				bits = c & ~seen[w];
				if (bits) {
					seen[w] |= bits;
					cur2[w] = bits;
				}
			}
		}
		const unsigned m = __ballot_sync(0xffffffffu, bits != 0);
		if (levels && m) {
			for (int k = 0; k < nroots; k++)
				if ((bits >> k) & 1ull) levels[(uint64_t)k * V + w] = (int32_t)depth1;
		}
		ws[r] = w;
		masks[r] = m;
		cnt += __popc(m);
		if (bits) e += __ldg(outdeg + w);
		any |= bits;
	}
#pragma unroll
	for (int o = 16; o > 0; o >>= 1) {
		e += __shfl_xor_sync(0xffffffffu, e, o);
		any |= __shfl_xor_sync(0xffffffffu, any, o);
	}
	if (lane == 0) {
		s_cnt[wid] = cnt;
		s_e[wid] = e;
		s_any[wid] = any;
	}
	__syncthreads();
	if (threadIdx.x == 0) {
		uint32_t tot = 0;
		unsigned long long et = 0;
		u64 at = 0;
		for (int x = 0; x < kWarps; x++) {
			const uint32_t c = s_cnt[x];
			s_cnt[x] = tot;
			tot += c;
			et += s_e[x];
			at |= s_any[x];
		}
		s_base = tot ? atomicAdd(ctr, (unsigned long long)tot) : 0ull;
		if (et) atomicAdd(ctr + 1, et);
		if (at) atomicOr(ctr + 2, at);
	}
	__syncthreads();
	unsigned long long pos = s_base + s_cnt[wid];
#pragma unroll
	for (int r = 0; r < kCommitPer; r++) {
		const unsigned m = masks[r];
		if ((m >> lane) & 1u) queue[pos + __popc(m & ((1u << lane) - 1u))] = ws[r];
		pos += __popc(m);
	}
}

__global__ void ms_clear(const uint32_t* queue, uint32_t n, u64* cur) {
	const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n) cur[__ldg(queue + i)] = 0;
}

// Per-root reached vertices and the out-degree sum over them, from the level
// rows: CTA column y takes root y's row (4 levels and 4 out-degrees per
// 16-byte load when the rows are aligned) and adds its block totals once.
// The out-degree array is read once per root, mostly from L2.
__global__ void ms_reach(const int32_t* levels, const uint32_t* outdeg, uint64_t V,
		unsigned long long* cnt, unsigned long long* edges) {
	__shared__ unsigned long long sc[8], se[8];
	const int k = blockIdx.y;
	const int32_t* row = levels + (uint64_t)k * V;
	const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
	uint64_t c = 0, e = 0;
	const bool vec = ((((uintptr_t)row) | ((uintptr_t)outdeg)) & 15u) == 0;
	uint64_t v0 = 0;
	if (vec) {
		const uint64_t nq = V / 4;
		for (uint64_t q = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; q < nq; q += stride) {
			const int4 l = __ldcs(reinterpret_cast<const int4*>(row) + q);
			const uint4 d = __ldg(reinterpret_cast<const uint4*>(outdeg) + q);
			if (l.x != kMsUnreached) { c++; e += d.x; }
			if (l.y != kMsUnreached) { c++; e += d.y; }
			if (l.z != kMsUnreached) { c++; e += d.z; }
			if (l.w != kMsUnreached) { c++; e += d.w; }
		}
		v0 = nq * 4;
	}
	for (uint64_t v = v0 + (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < V; v += stride)
		if (row[v] != kMsUnreached) { c++; e += __ldg(outdeg + v); }
#pragma unroll
	for (int o = 16; o > 0; o >>= 1) {
		c += __shfl_xor_sync(0xffffffffu, c, o);
		e += __shfl_xor_sync(0xffffffffu, e, o);
	}
	const uint32_t lane = threadIdx.x & 31u, wid = threadIdx.x >> 5;
	if (lane == 0) { sc[wid] = c; se[wid] = e; }
	__syncthreads();
	if (threadIdx.x == 0) {
		unsigned long long tc = 0, te = 0;
		for (uint32_t x = 0; x < (blockDim.x >> 5); x++) { tc += sc[x]; te += se[x]; }
		if (tc) atomicAdd(cnt + k, tc);
		if (te) atomicAdd(edges + k, te);
	}
}

// ---------------------------------------------------------------------------
// Batched Brandes betweenness centrality
//
// Reference: ll_b_bc_random (benchmark/benchmarks/bc_random.h:55-193): per
// source s, sigma is pushed along down edges (depth[w] == depth[v] + 1,
// ll_bfs_template.h:337-351) and the reverse sweep, deepest level first, sets
//   delta[v] = sum over down edges v->w of sigma[v] / sigma[w] * (1 + delta[w])
// and BC[v] += delta[v] for v != s (bc_random.h:73-111), in FP32 there and
// FP64 here.  A pass serves 64 sources: the BFS levels are the multi-source
// BFS above (lk[v] = the sources that have v at depth k, kept for every
// depth), and sigma / delta are 64 doubles per vertex.  An edge v->w is a
// down edge for exactly the sources in lk[v] & lk+1[w], so a sweep reads one
// 8-byte mask per edge and touches sigma and delta only for those sources:
// the work follows the (source, down edge) pairs, not 64 x every edge.  Both
// sweeps pull: sigma of level k + 1 over its vertices' in-edges, delta of
// level k over its vertices' out-edges, each vertex's sums kept in registers
// along its run of edges and added once per run (FP64 atomics only where a
// run is split between warps), so results agree with an exact evaluation to
// ~1e-15 relative, not bit for bit.  Without an in-CSR the sigma sweep
// pushes along out-edges instead, one atomic per (edge, source) pair.
// ---------------------------------------------------------------------------

// Sources of a pass: level-0 masks, sigma = 1, the sources' own-lane mask.
__global__ void bcm_roots(const int64_t* src, int n, u64* seen, u64* l0, u64* own,
		double* sigma, uint32_t* queue, unsigned long long* ctr, const uint32_t* outdeg) {
	const int k = threadIdx.x;
	if (k >= n) return;
	const uint32_t v = (uint32_t)src[k];
	atomicOr(seen + v, 1ull << k);
	atomicOr(own + v, 1ull << k);
	sigma[(uint64_t)v * kMsMaxRoots + k] = 1.0;
	const u64 old = atomicOr(l0 + v, 1ull << k);
	if (old == 0) {
		queue[atomicAdd(ctr, 1ull)] = v;
		atomicAdd(ctr + 1, (unsigned long long)__ldg(outdeg + v));
	}
}

// sigma[w][j] += sigma[v][j] over the out-edges v->w of level k's vertices
// for the sources j in lk[v] & lk1[w]; the warp takes such edges kMsBatch at
// a time (their sigma rows are loaded before any add, so the loads of the
// batch overlap), lane j serving sources j and j + 32.
constexpr int kMsBatch = 4;
__global__ void __launch_bounds__(kMsThreads)
bcm_sigma(SnapCsr out, const uint32_t* queue, const uint32_t* pos, uint32_t qlen,
		const u64* lk, const u64* lk1, double* sigma) {
	const uint32_t lane = threadIdx.x & 31u;
	const uint32_t total = __ldg(pos + qlen);
	const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
	const uint32_t range = ms_range(total, nwarps);
	const uint32_t nranges = (total + range - 1) / range;
	for (uint32_t r = warp; r < nranges; r += nwarps) {
		range_for_each(out, queue, pos, qlen, total, nranges, range, r,
			[&](bool act, uint32_t, uint32_t v, uint32_t w, uint32_t, uint32_t) {
				const u64 m = act ? (__ldg(lk + v) & __ldg(lk1 + w)) : 0ull;
				unsigned todo = __ballot_sync(0xffffffffu, m != 0);
				while (todo) {
					uint32_t tw[kMsBatch];
					bool b0[kMsBatch], b1[kMsBatch];
					double x0[kMsBatch], x1[kMsBatch];
#pragma unroll
					for (int u = 0; u < kMsBatch; u++) {
						const int t = todo ? __ffs(todo) - 1 : -1;   // warp-uniform
						todo &= todo - 1;
						tw[u] = 0;
						b0[u] = b1[u] = false;
						x0[u] = x1[u] = 0.0;
						if (t >= 0) {
							const uint32_t tv = __shfl_sync(0xffffffffu, v, t);
							tw[u] = __shfl_sync(0xffffffffu, w, t);
							const uint32_t lo = __shfl_sync(0xffffffffu, (uint32_t)m, t);
							const uint32_t hi = __shfl_sync(0xffffffffu, (uint32_t)(m >> 32), t);
							const double* sv = sigma + (uint64_t)tv * kMsMaxRoots;
							b0[u] = (lo >> lane) & 1u;
							b1[u] = (hi >> lane) & 1u;
							if (b0[u]) x0[u] = __ldcg(sv + lane);
							if (b1[u]) x1[u] = __ldcg(sv + 32 + lane);
						}
					}
#pragma unroll
					for (int u = 0; u < kMsBatch; u++) {
						double* sw = sigma + (uint64_t)tw[u] * kMsMaxRoots;
						if (b0[u]) atomicAdd(sw + lane, x0[u]);
						if (b1[u]) atomicAdd(sw + 32 + lane, x1[u]);
					}
				}
			});
	}
}

// The same sums pulled: for the vertices w of level k + 1's queue, over their
// in-edges v -> w (in-CSR ranges grouped by w), sigma[w][j] += sigma[v][j]
// for the sources j in lk[v] & lk1[w].  Each lane keeps w's two partial sums
// in registers over the run of w's in-edges and adds them to sigma[w] once
// per run, instead of one atomic per (edge, source) pair; kMsBatch edges'
// row loads are issued before their sums.
__global__ void __launch_bounds__(kMsThreads)
bcm_sigma_pull(SnapCsr in, const uint32_t* queue, const uint32_t* pos, uint32_t qlen,
		const u64* lk, const u64* lk1, double* sigma) {
	const uint32_t lane = threadIdx.x & 31u;
	const uint32_t total = __ldg(pos + qlen);
	const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
	const uint32_t range = ms_range(total, nwarps);
	const uint32_t nranges = (total + range - 1) / range;
	for (uint32_t r = warp; r < nranges; r += nwarps) {
		uint32_t cur = 0xffffffffu;
		double a0 = 0.0, a1 = 0.0;
		range_for_each(in, queue, pos, qlen, total, nranges, range, r,
			[&](bool act, uint32_t, uint32_t w, uint32_t v, uint32_t, uint32_t) {
				const u64 m = act ? (__ldg(lk + v) & __ldg(lk1 + w)) : 0ull;
				unsigned todo = __ballot_sync(0xffffffffu, m != 0);
				while (todo) {
					uint32_t tw[kMsBatch];
					double p0[kMsBatch], p1[kMsBatch];
#pragma unroll
					for (int u = 0; u < kMsBatch; u++) {
						const int t = todo ? __ffs(todo) - 1 : -1;   // warp-uniform
						todo &= todo - 1;
						tw[u] = 0xffffffffu;
						p0[u] = p1[u] = 0.0;
						if (t >= 0) {
							tw[u] = __shfl_sync(0xffffffffu, w, t);
							const uint32_t tv = __shfl_sync(0xffffffffu, v, t);
							const uint32_t lo = __shfl_sync(0xffffffffu, (uint32_t)m, t);
							const uint32_t hi = __shfl_sync(0xffffffffu, (uint32_t)(m >> 32), t);
							const double* sv = sigma + (uint64_t)tv * kMsMaxRoots;
							if ((lo >> lane) & 1u) p0[u] = __ldcg(sv + lane);
							if ((hi >> lane) & 1u) p1[u] = __ldcg(sv + 32 + lane);
						}
					}
#pragma unroll
					for (int u = 0; u < kMsBatch; u++) {
						if (tw[u] == 0xffffffffu) continue;          // warp-uniform
						if (tw[u] != cur) {
							if (cur != 0xffffffffu) {
								double* sw = sigma + (uint64_t)cur * kMsMaxRoots;
								if (a0 != 0.0) atomicAdd(sw + lane, a0);
								if (a1 != 0.0) atomicAdd(sw + 32 + lane, a1);
							}
							cur = tw[u];
							a0 = a1 = 0.0;
						}
						a0 += p0[u];
						a1 += p1[u];
					}
				}
			});
		if (cur != 0xffffffffu) {
			double* sw = sigma + (uint64_t)cur * kMsMaxRoots;
			if (a0 != 0.0) atomicAdd(sw + lane, a0);
			if (a1 != 0.0) atomicAdd(sw + 32 + lane, a1);
		}
	}
}

// delta[v][j] = sum over down edges v->w (j in lk[v] & lk1[w]) of
// sigma[v][j] * q[w][j], for level k's vertices, where q[w][j] =
// (1 + delta[w][j]) / sigma[w][j] has already replaced sigma[w][j] for the
// sources that have w at depth k + 1 (bcm_quot), so an edge costs an add, not
// a division: sigma[v][j] is the same for all of v's edges and multiplies
// the sum of q once per run.  Edges come grouped by v; each lane keeps v's
// two partial sums (sources j and j + 32) over the run and adds
// sigma[v][j] * sum to delta once per run; the q loads of kMsBatch edges are
// issued before their adds.
__device__ __forceinline__ void bcm_delta_flush(uint32_t v, double a0, double a1,
		const double* sigma, double* delta) {
	const uint32_t lane = threadIdx.x & 31u;
	const double* sv = sigma + (uint64_t)v * kMsMaxRoots;
	double* dv = delta + (uint64_t)v * kMsMaxRoots;
	if (a0 != 0.0) atomicAdd(dv + lane, __ldg(sv + lane) * a0);
	if (a1 != 0.0) atomicAdd(dv + 32 + lane, __ldg(sv + 32 + lane) * a1);
}

__global__ void __launch_bounds__(kMsThreads)
bcm_delta(SnapCsr out, const uint32_t* queue, const uint32_t* pos, uint32_t qlen,
		const u64* lk, const u64* lk1, const double* sigma, double* delta) {
	const uint32_t lane = threadIdx.x & 31u;
	const uint32_t total = __ldg(pos + qlen);
	const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
	const uint32_t range = ms_range(total, nwarps);
	const uint32_t nranges = (total + range - 1) / range;
	for (uint32_t r = warp; r < nranges; r += nwarps) {
		uint32_t cur = 0xffffffffu;
		double a0 = 0.0, a1 = 0.0;
		range_for_each(out, queue, pos, qlen, total, nranges, range, r,
			[&](bool act, uint32_t, uint32_t v, uint32_t w, uint32_t, uint32_t) {
				const u64 m = act ? (__ldg(lk + v) & __ldg(lk1 + w)) : 0ull;
				unsigned todo = __ballot_sync(0xffffffffu, m != 0);
				while (todo) {
					uint32_t tv[kMsBatch];
					double p0[kMsBatch], p1[kMsBatch];
#pragma unroll
					for (int u = 0; u < kMsBatch; u++) {
						const int t = todo ? __ffs(todo) - 1 : -1;   // warp-uniform
						todo &= todo - 1;
						tv[u] = 0xffffffffu;
						p0[u] = p1[u] = 0.0;
						if (t >= 0) {
							tv[u] = __shfl_sync(0xffffffffu, v, t);
							const uint32_t tw = __shfl_sync(0xffffffffu, w, t);
							const uint32_t lo = __shfl_sync(0xffffffffu, (uint32_t)m, t);
							const uint32_t hi = __shfl_sync(0xffffffffu, (uint32_t)(m >> 32), t);
							const double* qw = sigma + (uint64_t)tw * kMsMaxRoots;
							if ((lo >> lane) & 1u) p0[u] = __ldg(qw + lane);
							if ((hi >> lane) & 1u) p1[u] = __ldg(qw + 32 + lane);
						}
					}
#pragma unroll
					for (int u = 0; u < kMsBatch; u++) {
						if (tv[u] == 0xffffffffu) continue;          // warp-uniform
						if (tv[u] != cur) {
							if (cur != 0xffffffffu) bcm_delta_flush(cur, a0, a1, sigma, delta);
							cur = tv[u];
							a0 = a1 = 0.0;
						}
						a0 += p0[u];
						a1 += p1[u];
					}
				}
			});
		if (cur != 0xffffffffu) bcm_delta_flush(cur, a0, a1, sigma, delta);
	}
}

// For the vertices of a level whose delta is final: sigma[w][j] <-
// (1 + delta[w][j]) / sigma[w][j] for the sources j in lk[w] (the factor the
// level above multiplies by).  A warp per vertex, lane j serving j and j + 32.
__global__ void bcm_quot(const uint32_t* queue, uint32_t n, const u64* lk, double* sigma,
		const double* delta) {
	const uint32_t lane = threadIdx.x & 31u;
	const uint64_t i = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	if (i >= n) return;
	const uint32_t w = __ldg(queue + i);
	const u64 m = __ldg(lk + w);
	double* sw = sigma + (uint64_t)w * kMsMaxRoots;
	const double* dw = delta + (uint64_t)w * kMsMaxRoots;
	if ((m >> lane) & 1ull) sw[lane] = (1.0 + dw[lane]) / sw[lane];
	if ((m >> (lane + 32)) & 1ull) sw[32 + lane] = (1.0 + dw[32 + lane]) / sw[32 + lane];
}

// bc[v] += delta[v][j] over the sources j that reached v, v not being j's
// source, in increasing j.
__global__ void bcm_accum(const u64* seen, const u64* own, const double* delta, uint64_t V,
		double* bc) {
	const uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (v >= V) return;
	u64 b = seen[v] & ~own[v];
	if (!b) return;
	const double* dv = delta + v * kMsMaxRoots;
	double sum = 0.0;
	for (; b; b &= b - 1) sum += dv[__ffsll((long long)b) - 1];
	bc[v] += sum;
}

} // namespace lg

using namespace lg;

namespace {

// Grows b to hold `need` bytes keeping its first `keep` bytes.
lg_status grow_keep(DevBuf& b, size_t need, size_t keep, cudaStream_t st) {
	if (need <= b.bytes) return LG_OK;
	DevBuf nb;
	LG_TRY(nb.reserve(std::max(need, b.bytes * 2)));
	if (keep) LG_CUDA(cudaMemcpyAsync(nb.p, b.p, keep, cudaMemcpyDeviceToDevice, st), "grow");
	LG_CUDA(cudaStreamSynchronize(st), "grow");
	b.swap(nb);
	return LG_OK;
}

// The vertices of flat in-CSR f with more than `heavy` in-edges, listed in
// buf (a device counter, then the ids) for ms_bottom_up_heavy.
lg_status heavy_list(lg_store* s, const FlatCsr* f, uint64_t V, uint32_t heavy, DevBuf& buf,
		uint32_t** list, unsigned long long** count) {
	LG_TRY(buf.reserve(sizeof(unsigned long long) + std::max<uint64_t>(V, 1) * sizeof(uint32_t)));
	*count = buf.as<unsigned long long>();
	*list = reinterpret_cast<uint32_t*>(*count + 1);
	LG_CUDA(cudaMemsetAsync(*count, 0, sizeof(unsigned long long), s->stream), "clear");
	ms_heavy_list<<<grid_for(V, 256), 256, 0, s->stream>>>(f->off.as<uint32_t>(), (uint32_t)V,
			*list, *count, heavy);
	LG_CUDA(cudaGetLastError(), "ms_heavy_list");
	s->launches++;
	return LG_OK;
}

} // namespace

extern "C" lg_status lg_bc_batched(lg_snapshot* sn, const int64_t* sources, int n_sources,
		double* bc) {
	clear_error();
	if (!sn || !bc || (!sources && n_sources > 0)) return set_error(LG_EINVAL, "null argument");
	if (n_sources < 0) return set_error(LG_EINVAL, "negative source count");
	for (int i = 0; i < n_sources; i++)
		if (sources[i] < 0 || (uint64_t)sources[i] >= sn->V)
			return set_error(LG_EINVAL, "source %lld out of range", (long long)sources[i]);
	lg_store* s = sn->store;
	LG_CUDA(cudaSetDevice(s->device), "cudaSetDevice");
	cudaStream_t st = s->stream;
	const uint64_t V = sn->V;
	const unsigned B = 256;
	DevBuf* sc = s->scratch;
	LG_TRY(sc[0].reserve(3 * V * sizeof(u64)));                        // seen, nxt, own
	LG_TRY(sc[1].reserve(2 * V * kMsMaxRoots * sizeof(double)));       // sigma, delta
	LG_TRY(sc[3].reserve(V * sizeof(uint32_t)));                       // candidates
	LG_TRY(sc[5].reserve((2 * V + 1) * sizeof(uint32_t)));             // slot counts, prefix
	LG_TRY(sc[6].reserve(8 * sizeof(unsigned long long)));
	LG_TRY(sc[7].reserve(kMsMaxRoots * sizeof(int64_t)));
	u64* seen = sc[0].as<u64>();
	u64* nxt = seen + V;
	u64* own = nxt + V;
	double* sigma = sc[1].as<double>();
	double* delta = sigma + V * kMsMaxRoots;
	uint32_t* cand = sc[3].as<uint32_t>();
	uint32_t* qcnt = sc[5].as<uint32_t>();
	uint32_t* qpos = qcnt + V;
	unsigned long long* ctr = sc[6].as<unsigned long long>();
	DevBuf& masks = sc[2];          // level masks, V per level
	DevBuf& queues = sc[4];         // level queues, concatenated
	LG_TRY(grow_keep(masks, 8 * V * sizeof(u64), 0, st));
	LG_TRY(grow_keep(queues, 4 * V * sizeof(uint32_t), 0, st));
	const bool dev_out = is_device_pointer(bc);
	double* acc = bc;
	if (!dev_out) { LG_TRY(sc[8].reserve(V * sizeof(double))); acc = sc[8].as<double>(); }
	LG_CUDA(cudaMemsetAsync(acc, 0, V * sizeof(double), st), "clear bc");
	const FlatCsr* fi = sn->flat[1];
	const FlatCsr* fo = sn->flat[0];
	const SnapCsr out = (fo && fo->has_view) ? fo->view(sn->out.deg.as<uint32_t>()) : sn->view(0);
	const bool has_in = sn->in.present;
	const SnapCsr in = has_in ? sn->view(1) : out;
	if (!fi && has_in && n_sources > 0) {
		// the bottom-up steps read in-edges many times per pass: flatten them
		// for the call unless the snapshot already holds a flat in-CSR
		if (!s->flat_scratch) s->flat_scratch = new FlatCsr;
		LG_TRY(build_flat(sn, 1, *s->flat_scratch, false));
		fi = s->flat_scratch;
	}
	const uint32_t* outdeg = sn->out.deg.as<uint32_t>();
	int sms = 148;
	cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->device);
	const unsigned grid = (unsigned)sms * 8u;
	const double alpha = 14.0, beta = 24.0;
	uint32_t* hlist = nullptr;
	unsigned long long* hcount = nullptr;
	const uint32_t heavy = (uint32_t)tune_value(s->device, LG_TUNE_MS_HEAVY);
	if (fi) LG_TRY(heavy_list(s, fi, V, heavy, sc[10], &hlist, &hcount));

	for (int p0 = 0; p0 < n_sources; p0 += kMsMaxRoots) {
		const int n = std::min(kMsMaxRoots, n_sources - p0);
		const u64 lanes = n == 64 ? ~0ull : ((1ull << n) - 1ull);
		LG_CUDA(cudaMemsetAsync(seen, 0, 3 * V * sizeof(u64), st), "clear masks");
		LG_CUDA(cudaMemsetAsync(sigma, 0, 2 * V * kMsMaxRoots * sizeof(double), st), "clear");
		LG_CUDA(cudaMemsetAsync(masks.p, 0, 2 * V * sizeof(u64), st), "clear level masks");
		LG_CUDA(cudaMemsetAsync(ctr, 0, 8 * sizeof(unsigned long long), st), "clear counters");
		LG_CUDA(cudaMemcpyAsync(sc[7].p, sources + p0, n * sizeof(int64_t),
				cudaMemcpyHostToDevice, st), "sources");
		s->h2d_bytes += n * sizeof(int64_t);
		bcm_roots<<<1, kMsMaxRoots, 0, st>>>(sc[7].as<int64_t>(), n, seen, masks.as<u64>(), own,
				sigma, queues.as<uint32_t>(), ctr, outdeg);
		LG_CUDA(cudaGetLastError(), "bcm_roots");
		s->launches++;
		unsigned long long h[3];
		LG_TRY(read_words(s, ctr, 3, h));
		std::vector<uint64_t> qoff = {0, h[0]};   // level k's queue: [qoff[k], qoff[k+1])
		uint64_t mf = h[1];
		uint64_t mu = sn->out.n_edges > mf ? sn->out.n_edges - mf : 0;
		bool top_down = true;
		// forward: depths, then sigma, level by level
		for (uint32_t k = 0;; k++) {
			const uint64_t qb = qoff[k], qlen = qoff[k + 1] - qoff[k];
			if (qlen == 0) break;
			LG_TRY(grow_keep(masks, (uint64_t)(k + 3) * V * sizeof(u64),
					(uint64_t)(k + 2) * V * sizeof(u64), st));
			LG_TRY(grow_keep(queues, (qoff[k + 1] + V) * sizeof(uint32_t),
					qoff[k + 1] * sizeof(uint32_t), st));
			u64* lk = masks.as<u64>() + (uint64_t)k * V;
			u64* lk1 = lk + V;
			LG_CUDA(cudaMemsetAsync(lk1 + V, 0, V * sizeof(u64), st), "clear level masks");
			uint32_t* q = queues.as<uint32_t>() + qb;
			uint32_t* q2 = queues.as<uint32_t>() + qoff[k + 1];
			list_slots<<<grid_for(qlen, B), B, 0, st>>>(out, q, (uint32_t)qlen, qcnt);
			LG_TRY(exclusive_scan_u32(qcnt, qpos, qlen, sc[9], st, nullptr));
			if (top_down && has_in && (double)mf > (double)mu / alpha) top_down = false;
			else if (!top_down && (double)qlen < (double)V / beta) top_down = true;
			LG_CUDA(cudaMemsetAsync(ctr, 0, 4 * sizeof(unsigned long long), st), "memset");
			if (top_down) {
				ms_top_down<<<grid, kMsThreads, 0, st>>>(out, q, qpos, (uint32_t)qlen, lk, seen,
						nxt, cand, ctr + 3);
				unsigned long long nc = 0;
				LG_TRY(read_words(s, ctr + 3, 1, &nc));
				if (nc > 0)
					ms_commit<<<grid_for(nc, kMsThreads * kCommitPer), kMsThreads, 0, st>>>(cand,
							(uint32_t)nc, k + 1, V, n, nxt,
							seen, lk1, nullptr, outdeg, q2, ctr);
				s->launches += 5 + (nc > 0);
			} else {
				if (fi) {
					ms_bottom_up_flat<<<grid_for(V, kMsThreads * kMsVerts), kMsThreads, 0, st>>>(
							fi->off.as<uint32_t>(), fi->ids.as<uint32_t>(), (uint32_t)V, lanes,
							lk, seen, nxt, heavy);
					ms_bottom_up_heavy<<<grid, kMsThreads, 0, st>>>(fi->off.as<uint32_t>(),
							fi->ids.as<uint32_t>(), hlist, hcount, lanes, lk, seen, nxt);
					s->launches++;
				} else
					ms_bottom_up<<<grid_for(V, kMsThreads), kMsThreads, 0, st>>>(in, lanes, lk,
							seen, nxt);
				ms_commit<<<grid_for(V, kMsThreads * kCommitPer), kMsThreads, 0, st>>>(nullptr,
						(uint32_t)V, k + 1, V, n, nxt,
						seen, lk1, nullptr, outdeg, q2, ctr);
				s->launches += 5;
			}
			if (!has_in) {
				// push along the level's out-edges (one atomic per down pair)
				bcm_sigma<<<grid, kMsThreads, 0, st>>>(out, q, qpos, (uint32_t)qlen, lk, lk1,
						sigma);
				s->launches++;
			}
			LG_CUDA(cudaGetLastError(), "bc batched forward");
			LG_TRY(read_words(s, ctr, 3, h));
			if (has_in && h[0] > 0) {
				// pull into the new level over its in-edges
				list_slots<<<grid_for(h[0], B), B, 0, st>>>(in, q2, (uint32_t)h[0], qcnt);
				LG_TRY(exclusive_scan_u32(qcnt, qpos, h[0], sc[9], st, nullptr));
				bcm_sigma_pull<<<grid, kMsThreads, 0, st>>>(in, q2, qpos, (uint32_t)h[0], lk, lk1,
						sigma);
				LG_CUDA(cudaGetLastError(), "bc batched sigma");
				s->launches += 5;
			}
			qoff.push_back(qoff[k + 1] + h[0]);
			mf = h[1];
			mu -= std::min(mu, (uint64_t)mf);
		}
		// backward, deepest level with down edges first; level 0 holds only
		// the sources, whose own delta BC leaves out
		const int D = (int)qoff.size() - 1;           // levels 0 .. D-1 are non-empty
		for (int k = D - 1; k >= 1; k--) {
			const uint64_t qb = qoff[k], qlen = qoff[k + 1] - qoff[k];
			const u64* lk = masks.as<u64>() + (uint64_t)k * V;
			const uint32_t* q = queues.as<uint32_t>() + qb;
			if (k < D - 1) {                          // the deepest level has no down edges
				list_slots<<<grid_for(qlen, B), B, 0, st>>>(out, q, (uint32_t)qlen, qcnt);
				LG_TRY(exclusive_scan_u32(qcnt, qpos, qlen, sc[9], st, nullptr));
				bcm_delta<<<grid, kMsThreads, 0, st>>>(out, q, qpos, (uint32_t)qlen, lk, lk + V,
						sigma, delta);
				s->launches += 5;
			}
			if (k > 1) {                              // level k - 1 multiplies by these
				bcm_quot<<<grid_for(qlen * 32, B), B, 0, st>>>(q, (uint32_t)qlen, lk, sigma, delta);
				s->launches++;
			}
			LG_CUDA(cudaGetLastError(), "bc batched backward");
		}
		bcm_accum<<<grid_for(V, B), B, 0, st>>>(seen, own, delta, V, acc);
		LG_CUDA(cudaGetLastError(), "bcm_accum");
		s->launches++;
	}
	if (!dev_out) LG_TRY(copy_out(s, bc, acc, V * sizeof(double)));
	LG_CUDA(cudaStreamSynchronize(st), "bc batched");
	return LG_OK;
}

extern "C" lg_status lg_bfs_multi(lg_snapshot* sn, const int64_t* roots, int n_roots,
		int32_t* levels, lg_bfs_result* results) {
	clear_error();
	if (!sn || !roots || !levels) return set_error(LG_EINVAL, "null argument");
	if (n_roots <= 0) return set_error(LG_EINVAL, "n_roots must be positive");
	for (int k = 0; k < n_roots; k++)
		if (roots[k] < 0 || (uint64_t)roots[k] >= sn->V)
			return set_error(LG_EINVAL, "root %lld out of range", (long long)roots[k]);
	lg_store* s = sn->store;
	LG_CUDA(cudaSetDevice(s->device), "cudaSetDevice");
	cudaStream_t st = s->stream;
	const uint64_t V = sn->V;
	const unsigned B = 256;
	DevBuf* sc = s->scratch;
	LG_TRY(sc[0].reserve(2 * V * sizeof(u64)));            // seen, nxt
	LG_TRY(sc[1].reserve(2 * V * sizeof(u64)));            // cur, cur2
	LG_TRY(sc[2].reserve(2 * V * sizeof(uint32_t)));       // queue, next queue
	LG_TRY(sc[3].reserve(V * sizeof(uint32_t)));           // candidates
	LG_TRY(sc[5].reserve((2 * V + 1) * sizeof(uint32_t))); // slot counts, prefix
	LG_TRY(sc[6].reserve((8 + 2 * kMsMaxRoots) * sizeof(unsigned long long)));
	u64* seen = sc[0].as<u64>();
	u64* nxt = seen + V;
	u64* cur = sc[1].as<u64>();
	u64* cur2 = cur + V;
	uint32_t* q = sc[2].as<uint32_t>();
	uint32_t* q2 = q + V;
	uint32_t* cand = sc[3].as<uint32_t>();
	uint32_t* qcnt = sc[5].as<uint32_t>();
	uint32_t* qpos = qcnt + V;
	unsigned long long* ctr = sc[6].as<unsigned long long>();
	unsigned long long* lane_cnt = ctr + 8;
	unsigned long long* lane_edges = lane_cnt + kMsMaxRoots;
	const bool dev_out = is_device_pointer(levels);
	int32_t* lv = levels;
	if (!dev_out) {
		LG_TRY(sc[4].reserve((uint64_t)n_roots * V * sizeof(int32_t)));
		lv = sc[4].as<int32_t>();
	}
	// flat views where lg_snapshot_flatten made them
	const FlatCsr* fo = sn->flat[0];
	const FlatCsr* fi = sn->flat[1];
	const SnapCsr out = (fo && fo->has_view) ? fo->view(sn->out.deg.as<uint32_t>()) : sn->view(0);
	const bool has_in = sn->in.present;
	const SnapCsr in = has_in ? sn->view(1) : out;
	const uint32_t* outdeg = sn->out.deg.as<uint32_t>();
	int sms = 148;
	cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->device);
	const unsigned td_blocks = (unsigned)sms * 8u;
	const double alpha = 14.0, beta = 24.0;
	uint32_t* hlist = nullptr;
	unsigned long long* hcount = nullptr;
	const uint32_t heavy = (uint32_t)tune_value(s->device, LG_TUNE_MS_HEAVY);
	if (fi) LG_TRY(heavy_list(s, fi, V, heavy, sc[10], &hlist, &hcount));

	ms_fill<<<(unsigned)sms * 16u, B, 0, st>>>(lv, (uint64_t)n_roots * V);
	LG_CUDA(cudaGetLastError(), "ms_fill");
	s->launches++;
	for (int p0 = 0; p0 < n_roots; p0 += kMsMaxRoots) {
		const int n = std::min(kMsMaxRoots, n_roots - p0);
		const u64 lanes = n == 64 ? ~0ull : ((1ull << n) - 1ull);
		int32_t* plv = lv + (uint64_t)p0 * V;
		// (the previous pass swapped the pairs)
		cur = sc[1].as<u64>();
		cur2 = cur + V;
		q = sc[2].as<uint32_t>();
		q2 = q + V;
		LG_CUDA(cudaMemsetAsync(seen, 0, 2 * V * sizeof(u64), st), "clear masks");
		LG_CUDA(cudaMemsetAsync(cur, 0, 2 * V * sizeof(u64), st), "clear masks");
		LG_CUDA(cudaMemsetAsync(ctr, 0, (8 + 2 * kMsMaxRoots) * sizeof(unsigned long long), st),
				"clear counters");
		LG_TRY(sc[7].reserve(kMsMaxRoots * sizeof(int64_t)));
		LG_CUDA(cudaMemcpyAsync(sc[7].p, roots + p0, n * sizeof(int64_t),
				cudaMemcpyHostToDevice, st), "roots");
		s->h2d_bytes += n * sizeof(int64_t);
		ms_roots<<<1, kMsMaxRoots, 0, st>>>(sc[7].as<int64_t>(), n, V, outdeg, seen, cur, plv,
				q, ctr);
		LG_CUDA(cudaGetLastError(), "ms_roots");
		s->launches++;
		unsigned long long h[3];
		LG_TRY(read_words(s, ctr, 3, h));
		uint64_t qlen = h[0];
		uint64_t mf = h[1];        // out-degree sum of the frontier, for the direction choice
		uint64_t mu = sn->out.n_edges > mf ? sn->out.n_edges - mf : 0;
		int32_t depth = 0;
		int td = 0, bu = 0;
		std::vector<int32_t> maxlev(n, 0);
		bool top_down = true;
		while (qlen > 0) {
			if (top_down && has_in && (double)mf > (double)mu / alpha) top_down = false;
			else if (!top_down && (double)qlen < (double)V / beta) top_down = true;
			LG_CUDA(cudaMemsetAsync(ctr, 0, 4 * sizeof(unsigned long long), st), "memset");
			if (top_down) {
				list_slots<<<grid_for(qlen, B), B, 0, st>>>(out, q, (uint32_t)qlen, qcnt);
				LG_TRY(exclusive_scan_u32(qcnt, qpos, qlen, sc[8], st, nullptr));
				ms_top_down<<<td_blocks, kMsThreads, 0, st>>>(out, q, qpos, (uint32_t)qlen, cur,
						seen, nxt, cand, ctr + 3);
				unsigned long long nc = 0;
				LG_TRY(read_words(s, ctr + 3, 1, &nc));
				if (nc > 0)
					ms_commit<<<grid_for(nc, kMsThreads * kCommitPer), kMsThreads, 0, st>>>(cand,
							(uint32_t)nc, depth + 1, V, n, nxt,
							seen, cur2, plv, outdeg, q2, ctr);
				td++;
				s->launches += 5 + (nc > 0);
			} else {
				if (fi) {
					ms_bottom_up_flat<<<grid_for(V, kMsThreads * kMsVerts), kMsThreads, 0, st>>>(
							fi->off.as<uint32_t>(), fi->ids.as<uint32_t>(), (uint32_t)V, lanes,
							cur, seen, nxt, heavy);
					ms_bottom_up_heavy<<<td_blocks, kMsThreads, 0, st>>>(fi->off.as<uint32_t>(),
							fi->ids.as<uint32_t>(), hlist, hcount, lanes, cur, seen, nxt);
					s->launches++;
				} else
					ms_bottom_up<<<grid_for(V, kMsThreads), kMsThreads, 0, st>>>(in, lanes, cur,
							seen, nxt);
				ms_commit<<<grid_for(V, kMsThreads * kCommitPer), kMsThreads, 0, st>>>(nullptr,
						(uint32_t)V, depth + 1, V, n, nxt,
						seen, cur2, plv, outdeg, q2, ctr);
				bu++;
				s->launches += 2;
			}
			ms_clear<<<grid_for(qlen, B), B, 0, st>>>(q, (uint32_t)qlen, cur);
			LG_CUDA(cudaGetLastError(), "msbfs step");
			s->launches++;
			LG_TRY(read_words(s, ctr, 3, h));
			qlen = h[0];
			mf = h[1];
			mu -= std::min(mu, (uint64_t)mf);
			depth++;
			for (u64 b = h[2]; b; b &= b - 1) maxlev[__builtin_ctzll(b)] = depth;
			std::swap(q, q2);
			std::swap(cur, cur2);
		}
		if (results) {
			ms_reach<<<dim3((unsigned)sms * 2u, (unsigned)n), B, 0, st>>>(plv, outdeg, V,
					lane_cnt, lane_edges);
			LG_CUDA(cudaGetLastError(), "ms_reach");
			s->launches++;
			std::vector<unsigned long long> hc(2 * kMsMaxRoots);
			LG_CUDA(cudaMemcpyAsync(hc.data(), lane_cnt, hc.size() * sizeof(unsigned long long),
					cudaMemcpyDeviceToHost, st), "d2h");
			LG_CUDA(cudaStreamSynchronize(st), "msbfs");
			s->d2h_bytes += hc.size() * sizeof(unsigned long long);
			for (int k = 0; k < n; k++) {
				lg_bfs_result& r = results[p0 + k];
				r.reached = hc[k];
				r.reach_edges = hc[kMsMaxRoots + k];
				r.max_level = maxlev[k];
				r.top_down_steps = td;
				r.bottom_up_steps = bu;
				r.reserved = 0;
			}
		}
	}
	if (!dev_out) {
		LG_TRY(copy_out(s, levels, lv, (uint64_t)n_roots * V * sizeof(int32_t)));
		LG_CUDA(cudaStreamSynchronize(st), "msbfs");
	}
	return LG_OK;
}
