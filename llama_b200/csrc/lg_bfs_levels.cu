// lg_bfs_levels.cu - a whole direction-optimising BFS in one cooperative
// launch.
//
// lg_bfs's step-per-launch loop reads the next frontier's size back to the
// host after every level to choose the next direction, and a top-down level
// also reads its slot total for the range split: about a dozen host round
// trips per root, as long as the kernels themselves on an R-MAT scale-24
// snapshot.  bfs_levels runs every level inside one grid of co-resident CTAs
// (cudaLaunchCooperativeKernel) and replaces the round trips by grid
// barriers: each CTA reads the level's counters after the barrier and makes
// the same direction choice (the same rule and constants as the host loop),
// so the step sequence and the result equal lg_bfs's.
//
// Per level:
//   top-down   the frontier queue's slot counts and their exclusive scan are
//              formed in two barrier-separated phases (per-CTA sums, then
//              per-CTA offsets), then the balanced slot ranges of
//              lg_expand.cuh expand it; a vertex that wins its CAS is
//              appended to the next queue and set in the next frontier
//              bitmap.
//   bottom-up  only the rows of the flat in-CSR (vertices with in-edges) are
//              visited: after a top-down level all of them, reached ones
//              dropped; after a bottom-up level just the rows that level
//              left unfound, whose list it wrote.  On an R-MAT scale-24
//              snapshot 56 % of the vertices have no in-edges, and the
//              lists shrink level by level (7.4 M, 2.9 M, 0.08 M rows).  A
//              found vertex is set in the next frontier bitmap.  No queue is
//              built; a later top-down level first compacts the bitmap into
//              one.
// Counters rotate over three slots: level L reads slot L % 3 (filled during
// level L - 1), fills slot (L + 1) % 3 and clears slot (L + 2) % 3, which
// every CTA finished reading before the barrier that ended level L - 1.  The
// frontier bitmaps rotate the same way: level L reads bitmap L % 3, sets
// bits in (L + 1) % 3 and clears (L + 2) % 3, level L - 1's frontier, for
// level L + 1.
//
// Buffers written inside the kernel (queues, offsets, bitmaps, levels) are
// read through L2 or by plain loads after a barrier, never through the
// read-only path.  Every barrier wait is bounded (lg_coop.cuh: kCoopWaitNs of the global
// timer); a CTA that gives up sets an error flag, leaves, and the host
// reports LG_ETIMEOUT.
#include "lg_coop.cuh"
#include "lg_expand.cuh"
#include "lg_flat.cuh"
#include "lg_tune.h"

#include <mutex>

namespace lg {

namespace {

constexpr int kLvThreads = 512;
constexpr int kLvWarps = kLvThreads / 32;
constexpr int kLvVerts = 4;            // vertices a bottom-up thread interleaves
constexpr int kLvChunk = 4;            // in-neighbours per vertex per round
constexpr int kLvSmallPer = 4;         // queue entries per thread of the barrier-free scan
constexpr uint32_t kLvMaxRange = 1024; // top-down slots per warp range
constexpr int32_t kLvUnreached = LG_UNREACHED;
constexpr double kAlpha = 14.0, kBeta = 24.0;   // as lg_bfs's host loop

// Control block (device memory; bfs_levels_init resets it).
struct LvCtl {
	unsigned long long ctr[3][4];   // per level: [0] frontier size, [1] its out-degree
	                                // sum, [2] queue fill cursor, [3] unfound rows
	CoopBar bar;                    // err bit 0: a barrier wait gave up, bit 1: slots
	                                // above 2^32
	int32_t levels, td, bu, pad;
	unsigned long long reached, reach_edges;
};

// Appends item[j] for every j with take[j] to out at slots taken from *len:
// the CTA's count with one atomic, positions in (warp, j, lane) order.
// Every thread of the CTA calls it.
__device__ __forceinline__ void block_append_rows(const bool (&take)[kLvVerts],
		const uint32_t (&item)[kLvVerts], uint32_t* out, unsigned long long* len) {
	__shared__ uint32_t s_cnt[kLvWarps];
	__shared__ unsigned long long s_base;
	const uint32_t lane = threadIdx.x & 31u, wid = threadIdx.x >> 5;
	unsigned m[kLvVerts];
	uint32_t cnt = 0;
#pragma unroll
	for (int j = 0; j < kLvVerts; j++) {
		m[j] = __ballot_sync(0xffffffffu, take[j]);
		cnt += __popc(m[j]);
	}
	__syncthreads();                     // s_cnt / s_base free from a previous call
	if (lane == 0) s_cnt[wid] = cnt;
	__syncthreads();
	if (threadIdx.x == 0) {
		uint32_t tot = 0;
		for (int w = 0; w < kLvWarps; w++) {
			const uint32_t x = s_cnt[w];
			s_cnt[w] = tot;
			tot += x;
		}
		s_base = tot ? atomicAdd(len, (unsigned long long)tot) : 0ull;
	}
	__syncthreads();
	unsigned long long pos = s_base + s_cnt[wid];
	const unsigned below = (1u << lane) - 1u;
#pragma unroll
	for (int j = 0; j < kLvVerts; j++) {
		if (take[j]) out[pos + __popc(m[j] & below)] = item[j];
		pos += __popc(m[j]);
	}
}

__device__ __forceinline__ uint32_t lv_range(uint32_t total, uint32_t nwarps) {
	uint32_t r = (uint32_t)(((uint64_t)total + nwarps - 1) / nwarps);
	r = (r + 31u) & ~31u;
	return min(max(r, 32u), kLvMaxRange);
}

// Resets the control block and queues the root; bfs_levels fills the level
// array and the first two bitmaps itself.
__global__ void bfs_levels_init(uint32_t root, uint32_t* q0, const uint32_t* outdeg, LvCtl* c) {
	if (blockIdx.x == 0 && threadIdx.x == 0) {
		q0[0] = root;
		for (int i = 0; i < 3; i++)
			for (int j = 0; j < 4; j++) c->ctr[i][j] = 0;
		c->ctr[0][0] = 1;
		c->ctr[0][1] = __ldg(outdeg + root);
		c->bar.count = 0;
		c->bar.err = 0;
		c->levels = c->td = c->bu = c->pad = 0;
		c->reached = c->reach_edges = 0;
	}
}

// Two CTAs of 512 per SM: 64 registers, no spills.
__global__ void __launch_bounds__(kLvThreads, 2)
bfs_levels(SnapCsr out, const uint32_t* nz_rows, const uint32_t* nz_off, uint32_t R,
		uint32_t E, const uint32_t* in_ids, const uint32_t* outdeg, uint32_t V,
		unsigned long long out_edges, int has_in, int32_t* level, uint32_t* q0, uint32_t* q1,
		uint32_t* bits0, uint32_t* bits1, uint32_t* bits2, uint32_t* fcnt, uint32_t* fpos,
		unsigned long long* bsum, LvCtl* c) {
	const uint32_t W = (uint32_t)(((uint64_t)V + 31u) / 32u);
	const uint32_t tid = threadIdx.x, lane = tid & 31u;
	const uint32_t nthreads = gridDim.x * blockDim.x;
	const uint32_t gtid = blockIdx.x * blockDim.x + tid;
	const uint32_t nwarps = nthreads >> 5, gwarp = gtid >> 5;
	__shared__ uint32_t s_pos[kLvThreads * kLvSmallPer + 1];   // offsets of a small queue
	uint32_t *q = q0, *nq = q1;
	auto bm = [&](int i) { return i == 0 ? bits0 : i == 1 ? bits1 : bits2; };
	// every CTA keeps the same copy of the traversal state
	unsigned long long mu = out_edges, reached = 0, reach_edges = 0;
	bool top_down = true, have_queue = true;
	long long list_len = -1;          // unfound rows of the last bottom-up level, -1: none
	bool list_in_fcnt = false;        // that list is in fcnt (else in fpos)
	int32_t td = 0, bu = 0, cur = 0;
	{
		// levels: 0 at the root, unreached elsewhere; bitmap 0 = {root},
		// bitmap 1 clear (level 0's next frontier)
		const uint32_t root = __ldcg(q0);
		for (uint32_t v = gtid; v < V; v += nthreads) level[v] = v == root ? 0 : kLvUnreached;
		for (uint32_t w = gtid; w < W; w += nthreads) {
			bits0[w] = w == (root >> 5) ? 1u << (root & 31u) : 0u;
			bits1[w] = 0u;
		}
		if (!grid_barrier(&c->bar)) return;
	}
	for (;; cur++) {
		unsigned long long* now = c->ctr[cur % 3];
		unsigned long long* nxt = c->ctr[(cur + 1) % 3];
		// frontier bitmap, next frontier (cleared during the last level), and
		// the last level's frontier, cleared now for the next level
		uint32_t* bits = bm(cur % 3);
		uint32_t* nbits = bm((cur + 1) % 3);
		uint32_t* clear = bm((cur + 2) % 3);
		const unsigned long long qlen = __ldcg(now + 0), mf = __ldcg(now + 1);
		if (qlen == 0) break;
		reached += qlen;
		reach_edges += mf;
		mu -= min(mu, mf);
		if (top_down && has_in && (double)mf > (double)mu / kAlpha) top_down = false;
		else if (!top_down && (double)qlen < (double)V / kBeta) top_down = true;
		if (blockIdx.x == 0 && tid < 4) c->ctr[(cur + 2) % 3][tid] = 0;
		for (uint32_t w = gtid; w < W; w += nthreads) clear[w] = 0u;

		if (top_down) {
			if (!have_queue) {
				// the frontier is a bitmap: compact it into q (any order), one
				// counter atomic per CTA and round
				for (uint32_t b0 = blockIdx.x * blockDim.x; b0 < W; b0 += nthreads) {
					const uint32_t w = b0 + tid;
					const uint32_t m = w < W ? bits[w] : 0u;
					const uint32_t nb = __popc(m);
					uint32_t all;
					const uint32_t ex = block_exclusive_scan<kLvWarps>(nb, &all);
					__shared__ unsigned long long s_qbase;
					if (tid == 0) s_qbase = all ? atomicAdd(now + 2, (unsigned long long)all) : 0ull;
					__syncthreads();
					unsigned long long pos = s_qbase + ex;
					uint32_t mm = m;
					while (mm) {
						const int b = __ffs(mm) - 1;
						mm &= mm - 1u;
						q[pos++] = w * 32u + (uint32_t)b;
					}
				}
				if (!grid_barrier(&c->bar)) return;
				have_queue = true;
			}
			const uint32_t n = (uint32_t)qlen;
			unsigned long long tot = 0;
			const bool small = n <= (uint32_t)(kLvThreads * kLvSmallPer);
			if (small) {
				// a small queue: every CTA forms all the offsets itself in
				// shared memory, so no grid barrier is needed before expanding
				uint32_t kc[kLvSmallPer];
				unsigned long long sum = 0;
#pragma unroll
				for (int j = 0; j < kLvSmallPer; j++) {
					const uint32_t i = tid * kLvSmallPer + j;
					uint32_t f0;
					kc[j] = i < n ? vertex_slots(out, __ldcg(q + i), &f0) : 0u;
					sum += kc[j];
				}
				if (block_sum<kLvWarps>(sum) >= (1ull << 32)) {
					if (tid == 0) atomicOr(&c->bar.err, 2u);
					return;                      // every CTA sees the same total
				}
				uint32_t all;
				uint32_t ex = block_exclusive_scan<kLvWarps>((uint32_t)sum, &all);
#pragma unroll
				for (int j = 0; j < kLvSmallPer; j++) {
					const uint32_t i = tid * kLvSmallPer + j;
					if (i < n) s_pos[i] = ex;
					ex += kc[j];
				}
				if (tid == 0) s_pos[n] = all;
				tot = all;
				__syncthreads();
			} else {
				// phase A: slot counts of this CTA's share of the queue
				const uint32_t chunk = (n + gridDim.x - 1u) / gridDim.x;
				const uint32_t c0 = min(n, blockIdx.x * chunk), c1 = min(n, c0 + chunk);
				unsigned long long s = 0;
				for (uint32_t i = c0 + tid; i < c1; i += blockDim.x) {
					uint32_t f0;
					const uint32_t k = vertex_slots(out, __ldcg(q + i), &f0);
					fcnt[i] = k;
					s += k;
				}
				s = block_sum<kLvWarps>(s);
				if (tid == 0) bsum[blockIdx.x] = s;
				if (!grid_barrier(&c->bar)) return;
				// phase B: offsets (every CTA forms the same total)
				unsigned long long pre = 0;
				for (uint32_t b = tid; b < gridDim.x; b += blockDim.x) {
					const unsigned long long x = __ldcg(bsum + b);
					tot += x;
					if (b < blockIdx.x) pre += x;
				}
				pre = block_sum<kLvWarps>(pre);
				tot = block_sum<kLvWarps>(tot);
				if (tot >= (1ull << 32)) {
					if (tid == 0) atomicOr(&c->bar.err, 2u);
					return;                      // every CTA sees the same total
				}
				uint32_t run = (uint32_t)pre;
				for (uint32_t p = c0; p < c1; p += blockDim.x) {
					const uint32_t i = p + tid;
					const uint32_t x = i < c1 ? __ldcg(fcnt + i) : 0u;
					uint32_t piece;
					const uint32_t ex = block_exclusive_scan<kLvWarps>(x, &piece);
					if (i < c1) fpos[i] = run + ex;
					run += piece;
				}
				if (blockIdx.x == gridDim.x - 1u && tid == 0) fpos[n] = (uint32_t)tot;
				if (!grid_barrier(&c->bar)) return;
			}
			// phase C: expand the queue over balanced slot ranges
			const uint32_t total = (uint32_t)tot;
			const uint32_t range = lv_range(total, nwarps);
			const uint32_t nranges = (total + range - 1u) / range;
			unsigned long long mfn = 0;
			auto visit = [&](bool act, uint32_t, uint32_t, uint32_t w, uint32_t, uint32_t) {
				bool won = false;
				if (act && __ldcg(level + w) == kLvUnreached)
					won = atomicCAS(level + w, kLvUnreached, cur + 1) == kLvUnreached;
				const unsigned m = __ballot_sync(0xffffffffu, won);
				if (m) {
					const int leader = __ffs(m) - 1;
					unsigned long long b = 0;
					if ((int)lane == leader)
						b = atomicAdd(nxt + 0, (unsigned long long)__popc(m));
					b = __shfl_sync(0xffffffffu, b, leader);
					if (won) {
						nq[b + __popc(m & ((1u << lane) - 1u))] = w;
						atomicOr(nbits + (w >> 5), 1u << (w & 31u));
						mfn += __ldg(outdeg + w);
					}
				}
			};
			if (small) {
				for (uint32_t r = gwarp; r < nranges; r += nwarps)
					range_for_each<2>(out, q, s_pos, n, total, nranges, range, r, visit);
			} else {
				for (uint32_t r = gwarp; r < nranges; r += nwarps)
					range_for_each<1>(out, q, fpos, n, total, nranges, range, r, visit);
			}
			mfn = block_sum<kLvWarps>(mfn);
			if (tid == 0 && mfn) atomicAdd(nxt + 1, mfn);
			td++;
		} else {
			// bottom-up over the rows of the flat in-CSR that have in-edges:
			// all of them after a top-down level (dropping the reached ones),
			// else the previous bottom-up level's unfound rows.  A thread takes
			// kLvVerts rows and checks kLvChunk in-neighbours of each per
			// round; the rows still unfound form the next level's list.
			const bool from_list = list_len >= 0;
			const uint32_t* lin = list_in_fcnt ? fcnt : fpos;
			uint32_t* lout = list_in_fcnt ? fpos : fcnt;
			const uint32_t items = from_list ? (uint32_t)list_len : R;
			unsigned long long mfn = 0, cnt = 0;
			for (uint32_t base = blockIdx.x * (uint32_t)(kLvThreads * kLvVerts); base < items;
					base += nthreads * (uint32_t)kLvVerts) {
				uint32_t k[kLvVerts], end[kLvVerts], row[kLvVerts], v[kLvVerts];
				bool found[kLvVerts], keep[kLvVerts];
#pragma unroll
				for (int j = 0; j < kLvVerts; j++) {
					const uint32_t i = base + j * kLvThreads + tid;
					row[j] = 0; v[j] = 0; k[j] = 0; end[j] = 0;
					found[j] = false; keep[j] = false;
					if (i < items) {
						row[j] = from_list ? __ldcg(lin + i) : i;
						v[j] = __ldg(nz_rows + row[j]);
						k[j] = __ldg(nz_off + row[j]);
						end[j] = row[j] + 1 < R ? __ldg(nz_off + row[j] + 1) : E;
						keep[j] = true;
					}
				}
				if (!from_list) {
#pragma unroll
					for (int j = 0; j < kLvVerts; j++)
						if (keep[j] && __ldcg(level + v[j]) != kLvUnreached) {
							keep[j] = false;
							end[j] = k[j];
						}
				}
				bool more = true;
				while (more) {
					uint32_t u[kLvVerts][kLvChunk], wd[kLvVerts][kLvChunk];
#pragma unroll
					for (int j = 0; j < kLvVerts; j++)
#pragma unroll
						for (int x = 0; x < kLvChunk; x++)
							u[j][x] = k[j] + x < end[j] ? __ldg(in_ids + k[j] + x) : kNoId;
#pragma unroll
					for (int j = 0; j < kLvVerts; j++)
#pragma unroll
						for (int x = 0; x < kLvChunk; x++)
							wd[j][x] = u[j][x] != kNoId ? bits[u[j][x] >> 5] : 0u;
					more = false;
#pragma unroll
					for (int j = 0; j < kLvVerts; j++) {
						bool hit = false;
#pragma unroll
						for (int x = 0; x < kLvChunk; x++)
							hit |= ((wd[j][x] >> (u[j][x] & 31u)) & 1u) != 0;
						if (hit) { found[j] = true; k[j] = end[j]; }
						else k[j] = min(k[j] + kLvChunk, end[j]);
						more |= k[j] < end[j];
					}
				}
#pragma unroll
				for (int j = 0; j < kLvVerts; j++) {
					if (__any_sync(0xffffffffu, found[j])) {
						// lanes whose vertices share a bitmap word OR their bits
						// into one atomic (rows are in vertex order, so they
						// often do)
						const uint32_t wv = found[j] ? v[j] >> 5 : 0xffffffffu;
						const unsigned grp = __match_any_sync(0xffffffffu, wv);
						const uint32_t orv = __reduce_or_sync(grp,
								found[j] ? 1u << (v[j] & 31u) : 0u);
						if (found[j]) {
							level[v[j]] = cur + 1;
							if ((int)lane == __ffs(grp) - 1) atomicOr(nbits + wv, orv);
							mfn += __ldg(outdeg + v[j]);
							cnt++;
						}
					}
				}
				// unfound rows: the next bottom-up level's list, one counter
				// atomic per CTA and round
				bool stay[kLvVerts];
#pragma unroll
				for (int j = 0; j < kLvVerts; j++) stay[j] = keep[j] && !found[j];
				block_append_rows(stay, row, lout, nxt + 3);
			}
			cnt = block_sum<kLvWarps>(cnt);
			mfn = block_sum<kLvWarps>(mfn);
			if (tid == 0) {
				if (cnt) atomicAdd(nxt + 0, cnt);
				if (mfn) atomicAdd(nxt + 1, mfn);
			}
			bu++;
		}
		if (!grid_barrier(&c->bar)) return;
		if (top_down) {
			uint32_t* t = q; q = nq; nq = t;
			have_queue = true;
			list_len = -1;                 // fcnt / fpos were overwritten
		} else {
			have_queue = false;
			list_len = (long long)__ldcg(nxt + 3);
			list_in_fcnt = !list_in_fcnt;
		}
	}
	if (blockIdx.x == 0 && tid == 0) {
		c->levels = cur;
		c->td = td;
		c->bu = bu;
		c->reached = reached;
		c->reach_edges = reach_edges;
	}
}

std::mutex g_coop_mu;
int g_coop[LG_TUNE_MAX_DEVICES];          // co-resident CTAs of bfs_levels + 1, 0 = not probed

int coop_grid(int device) {
	std::lock_guard<std::mutex> lk(g_coop_mu);
	if (device < 0 || device >= LG_TUNE_MAX_DEVICES) return 0;
	if (!g_coop[device])
		g_coop[device] = 1 + coop_grid_size((const void*)bfs_levels, kLvThreads, device);
	return g_coop[device] - 1;
}

} // namespace

// One cooperative launch for the whole BFS from `root` into device array lvl
// (lg_bfs's contract).  *ran = false, and nothing is launched, when the
// snapshot's in-CSR is kept but not flat, LG_TUNE_BFS_LEVELS is 0, or the
// device has no cooperative launch; the caller then runs its per-level loop.
lg_status bfs_levels_run(lg_snapshot* sn, uint32_t root, int32_t* lvl, lg_bfs_result* result,
		bool* ran) {
	*ran = false;
	lg_store* s = sn->store;
	const FlatCsr* fi = sn->flat[1];
	if (sn->in.present && !fi) return LG_OK;
	if (!tune_value(s->device, LG_TUNE_BFS_LEVELS)) return LG_OK;
	const int grid = coop_grid(s->device);
	if (grid <= 0) return LG_OK;
	cudaStream_t st = s->stream;
	const uint64_t V = sn->V;
	const uint64_t W = (V + 31) / 32;
	DevBuf* sc = s->scratch;
	LG_TRY(sc[0].reserve(V * 4));
	LG_TRY(sc[1].reserve(V * 4));
	LG_TRY(sc[2].reserve(W * 4));
	LG_TRY(sc[8].reserve(W * 4));
	LG_TRY(sc[10].reserve(W * 4));
	LG_TRY(sc[5].reserve(V * 4));
	LG_TRY(sc[6].reserve((V + 1) * 4));
	LG_TRY(sc[9].reserve(sizeof(LvCtl) + (size_t)grid * sizeof(unsigned long long)));
	const FlatCsr* fo = sn->flat[0];
	SnapCsr out = (fo && fo->has_view) ? fo->view(sn->out.deg.as<uint32_t>()) : sn->view(0);
	const uint32_t* nz_rows = fi ? fi->nz_rows() : nullptr;
	const uint32_t* nz_off = fi ? fi->nz_off() : nullptr;
	uint32_t R = fi ? (uint32_t)fi->R : 0u, E = fi ? (uint32_t)fi->E : 0u;
	const uint32_t* in_ids = fi ? fi->ids.as<uint32_t>() : nullptr;
	const uint32_t* outdeg = sn->out.deg.as<uint32_t>();
	uint32_t V32 = (uint32_t)V;
	unsigned long long out_edges = sn->out.n_edges;
	int has_in = sn->in.present ? 1 : 0;
	uint32_t* q0 = sc[0].as<uint32_t>();
	uint32_t* q1 = sc[1].as<uint32_t>();
	uint32_t* bits0 = sc[2].as<uint32_t>();
	uint32_t* bits1 = sc[8].as<uint32_t>();
	uint32_t* bits2 = sc[10].as<uint32_t>();
	uint32_t* fcnt = sc[5].as<uint32_t>();
	uint32_t* fpos = sc[6].as<uint32_t>();
	LvCtl* ctl = sc[9].as<LvCtl>();
	unsigned long long* bsum = reinterpret_cast<unsigned long long*>(
			sc[9].as<unsigned char>() + sizeof(LvCtl));
	bfs_levels_init<<<1, 32, 0, st>>>(root, q0, outdeg, ctl);
	LG_CUDA(cudaGetLastError(), "bfs_levels_init");
	void* args[] = {&out, &nz_rows, &nz_off, &R, &E, &in_ids, &outdeg, &V32, &out_edges,
			&has_in, &lvl, &q0, &q1, &bits0, &bits1, &bits2, &fcnt, &fpos, &bsum, &ctl};
	LG_CUDA(cudaLaunchCooperativeKernel((const void*)bfs_levels, dim3((unsigned)grid),
			dim3(kLvThreads), args, 0, st), "bfs_levels");
	s->launches += 2;
	LvCtl h;
	LG_CUDA(cudaMemcpyAsync(&h, ctl, sizeof(h), cudaMemcpyDeviceToHost, st), "d2h");
	LG_CUDA(cudaStreamSynchronize(st), "bfs_levels");
	s->d2h_bytes += sizeof(h);
	if (h.bar.err & 1u)
		return set_error(LG_ETIMEOUT, "bfs: a grid barrier wait ran out (%d levels done)",
				h.levels);
	if (h.bar.err & 2u)
		return set_error(LG_ENOTSUP, "bfs: a frontier holds 2^32 or more slots");
	if (result) {
		result->reached = h.reached;
		result->reach_edges = h.reach_edges;
		result->max_level = h.levels - 1;
		result->top_down_steps = h.td;
		result->bottom_up_steps = h.bu;
		result->reserved = 0;
	}
	*ran = true;
	return LG_OK;
}

} // namespace lg
