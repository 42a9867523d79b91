// lg_bfs.cu - breadth-first search levels over a snapshot.
//
// Reference: ll_bfs_template (llama/include/llama/ll_bfs_template.h:152-293)
// driven by u_sssp_bfs / ll_b_sssp_unweighted_bfs
// (benchmark/benchmarks/sssp.h:219-300): level-synchronous, top-down only,
// dist[root] = 0, unreached vertices keep INT_MAX - 1.  BFS levels are
// unique, so any level-synchronous traversal yields the same array; this one
// is direction-optimising (Beamer et al., SC'12): top-down steps expand the
// frontier queue over the out-CSR in balanced slot ranges, bottom-up steps let every
// unvisited vertex look for a parent among its in-neighbours (in-CSR) in a
// frontier bitmap that stays resident in L2.
#include "lg_expand.cuh"
#include "lg_flat.cuh"

namespace lg {

// lg_bfs_levels.cu: the whole BFS in one cooperative launch; *ran = false
// when it does not apply to the snapshot (nothing launched).
lg_status bfs_levels_run(lg_snapshot* sn, uint32_t root, int32_t* lvl, lg_bfs_result* result,
		bool* ran);

constexpr int32_t kUnreached = LG_UNREACHED;
constexpr int kBfsThreads = 256;
constexpr uint32_t kBfsRange = 1024;
constexpr uint64_t kBfsWarps = 148ull * 64;   // about the warps a B200 holds at once
constexpr int kBuChunk = 4;            // in-neighbours a bottom-up round checks
constexpr int kBuVerts = 4;            // vertices a flat bottom-up thread interleaves

__global__ void bfs_init(int32_t* level, uint64_t V, uint32_t root,
		uint32_t* queue, const uint32_t* outdeg, unsigned long long* ctr) {
	uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (v < V) level[v] = (v == root) ? 0 : kUnreached;
	if (v == 0) {
		queue[0] = root;
		ctr[0] = 0;
		ctr[1] = outdeg[root];
	}
}

// Warp-aggregated append of `item` for the lanes with `take` set; returns
// the number of items the warp appended.
__device__ __forceinline__ void warp_append(bool take, uint32_t item,
		uint32_t* queue, unsigned long long* len) {
	unsigned m = __ballot_sync(0xffffffffu, take);
	if (!m) return;
	const uint32_t lane = threadIdx.x & 31u;
	const int leader = __ffs(m) - 1;
	unsigned long long base = 0;
	if ((int)lane == leader) base = atomicAdd(len, (unsigned long long)__popc(m));
	base = __shfl_sync(0xffffffffu, base, leader);
	if (take) queue[base + __popc(m & ((1u << lane) - 1u))] = item;
}

__device__ __forceinline__ void warp_add_u64(unsigned long long x,
		unsigned long long* dst) {
	for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
	if ((threadIdx.x & 31) == 0 && x) atomicAdd(dst, x);
}

// Block-aggregated append for the dense steps, which visit every vertex:
// each thread offers N items (take[j], item[j]) and adds `sum` to len[1];
// the block takes its queue slots with one atomic on len[0] and adds its
// sum with one more, instead of two atomics per warp on the same counters.
// Every thread of the block (kBfsThreads) calls it.
template <int N>
__device__ __forceinline__ void block_append(const bool (&take)[N], const uint32_t (&item)[N],
		unsigned long long sum, uint32_t* queue, unsigned long long* len) {
	constexpr int kWarps = kBfsThreads / 32;
	__shared__ uint32_t s_cnt[kWarps];
	__shared__ unsigned long long s_sum[kWarps];
	__shared__ unsigned long long s_base;
	const uint32_t lane = threadIdx.x & 31u, wid = threadIdx.x >> 5;
	unsigned m[N];
	uint32_t cnt = 0;
#pragma unroll
	for (int j = 0; j < N; j++) {
		m[j] = __ballot_sync(0xffffffffu, take[j]);
		cnt += __popc(m[j]);
	}
#pragma unroll
	for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
	if (lane == 0) {
		s_cnt[wid] = cnt;
		s_sum[wid] = sum;
	}
	__syncthreads();
	if (threadIdx.x == 0) {
		uint32_t tot = 0;
		unsigned long long st = 0;
		for (int x = 0; x < kWarps; x++) {
			const uint32_t c = s_cnt[x];
			s_cnt[x] = tot;
			tot += c;
			st += s_sum[x];
		}
		s_base = tot ? atomicAdd(len, (unsigned long long)tot) : 0ull;
		if (st) atomicAdd(len + 1, st);
	}
	__syncthreads();
	unsigned long long pos = s_base + s_cnt[wid];
	const unsigned below = (1u << lane) - 1u;
#pragma unroll
	for (int j = 0; j < N; j++) {
		if (take[j]) queue[pos + __popc(m[j] & below)] = item[j];
		pos += __popc(m[j]);
	}
}

// Fragment slots of every frontier entry (to be scanned into range offsets).
__global__ void bfs_frontier_slots(SnapCsr out, const uint32_t* queue, uint32_t qlen,
		uint32_t* cnt) {
	const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= qlen) return;
	uint32_t f0;
	cnt[i] = vertex_slots(out, __ldg(queue + i), &f0);
}

// Top-down step over the frontier's slot space cut into ranges of at most
// kBfsRange slots, one warp each (lg_expand.cuh).  ctr[0] = next frontier size,
// ctr[1] = sum of out-degrees of the next frontier.
__global__ void __launch_bounds__(kBfsThreads)
bfs_top_down(SnapCsr out, const uint32_t* queue, const uint32_t* fpos, uint32_t qlen,
		uint32_t total, uint32_t range, uint32_t nranges, int32_t* level, uint32_t* next,
		unsigned long long* ctr, int32_t cur) {
	const uint32_t lane = threadIdx.x & 31u;
	const uint64_t r64 = (uint64_t)blockIdx.x * (kBfsThreads / 32) + (threadIdx.x >> 5);
	if (r64 >= nranges) return;
	const uint32_t r = (uint32_t)r64;
	const bool last_range = r == nranges - 1;
	const uint32_t ra = r * range;
	const uint32_t rb = last_range ? total : min(total, ra + range);
	uint32_t e_begin, e_end;
	range_entries(fpos, qlen, ra, rb, last_range, &e_begin, &e_end);
	const LevelTab* lt = out.lt;
	unsigned long long mf = 0;
	for (uint32_t ew = e_begin; ew < e_end; ew += 32) {
		const Window w = load_window(out, queue, fpos, ew, e_end, ra, rb);
		for (uint32_t base = w.lo; base < w.hi; base += 32 * kUnroll) {
			uint32_t nb[kUnroll];
			bool act[kUnroll];
#pragma unroll
			for (int u = 0; u < kUnroll; u++) {
				const uint32_t k = base + u * 32 + lane;
				uint32_t own, lv, idx;
				locate_slot(out, w, k, &own, &lv, &idx);
				act[u] = k < w.hi;
				nb[u] = 0;
				if (act[u]) {
					const uint32_t word = __ldg(lt->del[lv] + (idx >> 5));
					nb[u] = __ldg(lt->ids[lv] + idx);
					act[u] = !((word >> (idx & 31)) & 1u);
				}
			}
			int32_t seen[kUnroll];
#pragma unroll
			for (int u = 0; u < kUnroll; u++) seen[u] = act[u] ? __ldcg(level + nb[u]) : 0;
#pragma unroll
			for (int u = 0; u < kUnroll; u++) {
				bool won = false;
				if (act[u] && seen[u] == kUnreached)
					won = atomicCAS(level + nb[u], kUnreached, cur + 1) == kUnreached;
				warp_append(won, nb[u], next, ctr);
				if (won) mf += __ldg(out.deg + nb[u]);
			}
		}
	}
	warp_add_u64(mf, ctr + 1);
}

__global__ void bfs_set_bits(const uint32_t* queue, uint32_t qlen, uint32_t* bits) {
	uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= qlen) return;
	uint32_t u = queue[i];
	atomicOr(bits + (u >> 5), 1u << (u & 31));
}

__global__ void __launch_bounds__(kBfsThreads)
bfs_bottom_up(SnapCsr in, const uint32_t* outdeg, const uint32_t* bits,
		int32_t* level, uint32_t* next, unsigned long long* ctr, int32_t cur) {
	const uint64_t v64 = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	const uint32_t v = (uint32_t)v64;
	bool found = false;
	if (v64 < in.V && level[v] == kUnreached) {
		const uint32_t f0 = __ldg(in.frag_off + v), f1 = __ldg(in.frag_off + v + 1);
		for (uint32_t f = f0; f < f1 && !found; f++) {
			const uint2 fr = in.frags[f];
			const uint32_t lv = frag_level(fr), n = frag_len(fr);
			const uint32_t* ids = in.lt->ids[lv] + fr.x;
			// kBuChunk neighbours per round: their id and bitmap loads are
			// independent, so a round costs two memory latencies, not 2 x kBuChunk
			for (uint32_t k = 0; k < n && !found; k += kBuChunk) {
				uint32_t u[kBuChunk], w[kBuChunk];
#pragma unroll
				for (int j = 0; j < kBuChunk; j++)
					u[j] = k + j < n ? __ldg(ids + k + j) : kNoId;
#pragma unroll
				for (int j = 0; j < kBuChunk; j++)
					w[j] = u[j] != kNoId ? __ldg(bits + (u[j] >> 5)) : 0u;
#pragma unroll
				for (int j = 0; j < kBuChunk; j++) {
					if (!found && ((w[j] >> (u[j] & 31u)) & 1u)
							&& !slot_deleted(in.lt, lv, fr.x + k + j))
						found = true;
				}
			}
		}
		if (found) level[v] = cur + 1;
	}
	const bool take[1] = {found};
	const uint32_t item[1] = {v};
	block_append(take, item, found ? __ldg(outdeg + v) : 0ull, next, ctr);
}

// Bottom-up step over a flat in-CSR (lg_snapshot_flatten).  A thread takes
// kBuVerts vertices (kBfsThreads apart, so the level and offset loads stay
// coalesced) and checks kBuChunk in-neighbours of each of them per round:
// up to kBuVerts x kBuChunk id loads, then as many bitmap loads, in flight
// at once.  No deletion bits: the flat CSR holds live edges only.
__global__ void __launch_bounds__(kBfsThreads)
bfs_bottom_up_flat(const uint32_t* off, const uint32_t* ids, uint32_t V,
		const uint32_t* outdeg, const uint32_t* bits, int32_t* level,
		uint32_t* next, unsigned long long* ctr, int32_t cur) {
	const uint32_t base = blockIdx.x * (uint32_t)(kBfsThreads * kBuVerts) + threadIdx.x;
	uint32_t k[kBuVerts], end[kBuVerts];
	bool found[kBuVerts];
#pragma unroll
	for (int j = 0; j < kBuVerts; j++) {
		const uint32_t v = base + j * kBfsThreads;
		k[j] = 0; end[j] = 0; found[j] = false;
		if (v < V && level[v] == kUnreached) { k[j] = __ldg(off + v); end[j] = __ldg(off + v + 1); }
	}
	bool more = true;
	while (more) {
		uint32_t u[kBuVerts][kBuChunk], w[kBuVerts][kBuChunk];
#pragma unroll
		for (int j = 0; j < kBuVerts; j++)
#pragma unroll
			for (int c = 0; c < kBuChunk; c++)
				u[j][c] = k[j] + c < end[j] ? __ldg(ids + k[j] + c) : kNoId;
#pragma unroll
		for (int j = 0; j < kBuVerts; j++)
#pragma unroll
			for (int c = 0; c < kBuChunk; c++)
				w[j][c] = u[j][c] != kNoId ? __ldg(bits + (u[j][c] >> 5)) : 0u;
		more = false;
#pragma unroll
		for (int j = 0; j < kBuVerts; j++) {
			bool hit = false;
#pragma unroll
			for (int c = 0; c < kBuChunk; c++) hit |= ((w[j][c] >> (u[j][c] & 31u)) & 1u) != 0;
			if (hit) { found[j] = true; k[j] = end[j]; }
			else k[j] = min(k[j] + kBuChunk, end[j]);
			more |= k[j] < end[j];
		}
	}
	unsigned long long mf = 0;
	uint32_t item[kBuVerts];
#pragma unroll
	for (int j = 0; j < kBuVerts; j++) {
		const uint32_t v = base + j * kBfsThreads;
		item[j] = v;
		if (found[j]) { level[v] = cur + 1; mf += __ldg(outdeg + v); }
	}
	block_append(found, item, mf, next, ctr);
}

} // namespace lg

using namespace lg;

extern "C" lg_status lg_bfs(lg_snapshot* sn, int64_t root, int32_t* levels,
		lg_bfs_result* result) {
	clear_error();
	if (!sn || !levels) return set_error(LG_EINVAL, "null argument");
	if (root < 0 || (uint64_t)root >= sn->V)
		return set_error(LG_EINVAL, "root %lld out of range", (long long)root);
	lg_store* s = sn->store;
	LG_CUDA(cudaSetDevice(s->device), "cudaSetDevice");
	cudaStream_t st = s->stream;
	const uint64_t V = sn->V;
	DevBuf* sc = s->scratch;
	LG_TRY(sc[0].reserve(V * 4));
	LG_TRY(sc[1].reserve(V * 4));
	LG_TRY(sc[2].reserve(((V + 31) / 32) * 4));
	LG_TRY(sc[3].reserve(4 * sizeof(unsigned long long)));
	LG_TRY(sc[5].reserve(V * 4));
	LG_TRY(sc[6].reserve((V + 1) * 4));
	uint32_t* fcnt = sc[5].as<uint32_t>();
	uint32_t* fpos = sc[6].as<uint32_t>();
	const bool dev_out = is_device_pointer(levels);
	int32_t* lvl = levels;
	if (!dev_out) {
		LG_TRY(sc[4].reserve(V * 4));
		lvl = sc[4].as<int32_t>();
	}
	// the whole traversal in one cooperative launch where it applies
	bool ran = false;
	LG_TRY(bfs_levels_run(sn, (uint32_t)root, lvl, result, &ran));
	if (ran) {
		if (!dev_out) {
			LG_TRY(copy_out(s, levels, lvl, V * 4));
			LG_CUDA(cudaStreamSynchronize(st), "bfs");
		}
		return LG_OK;
	}
	uint32_t* q = sc[0].as<uint32_t>();
	uint32_t* nq = sc[1].as<uint32_t>();
	uint32_t* bits = sc[2].as<uint32_t>();
	unsigned long long* ctr = sc[3].as<unsigned long long>();
	// flat views where lg_snapshot_flatten made them
	const FlatCsr* fo = sn->flat[0];
	const FlatCsr* fi = sn->flat[1];
	const SnapCsr out = (fo && fo->has_view) ? fo->view(sn->out.deg.as<uint32_t>()) : sn->view(0);
	const SnapCsr in = sn->in.present ? sn->view(1) : out;
	const uint32_t* outdeg = sn->out.deg.as<uint32_t>();

	bfs_init<<<grid_for(V, 256), 256, 0, st>>>(lvl, V, (uint32_t)root, q, outdeg, ctr);
	LG_CUDA(cudaGetLastError(), "bfs_init");
	s->launches++;
	unsigned long long h[2];
	LG_TRY(read_words(s, ctr, 2, h));
	uint64_t qlen = 1, mf = h[1];
	uint64_t mu = sn->out.n_edges - mf;   // edges out of unvisited vertices
	uint64_t reached = 1, reach_edges = mf;
	int32_t cur = 0;
	int td_steps = 0, bu_steps = 0;
	bool top_down = true;
	const double alpha = 14.0, beta = 24.0;
	while (qlen > 0) {
		if (top_down && sn->in.present && (double)mf > (double)mu / alpha)
			top_down = false;
		else if (!top_down && (double)qlen < (double)V / beta)
			top_down = true;
		LG_CUDA(cudaMemsetAsync(ctr, 0, 2 * sizeof(unsigned long long), st), "memset");
		if (top_down) {
			// frontier slot offsets, then one warp per range
			bfs_frontier_slots<<<grid_for(qlen, 256), 256, 0, st>>>(out, q,
					(uint32_t)qlen, fcnt);
			uint64_t total = 0;
			LG_TRY(exclusive_scan_u32(fcnt, fpos, qlen, sc[7], st, &total));
			s->d2h_bytes += 8;
			// ranges of up to kBfsRange slots, shorter (down to 32) when the
			// frontier is too small to give every resident warp one
			uint64_t range = (total + kBfsWarps - 1) / kBfsWarps;
			range = std::min<uint64_t>(std::max<uint64_t>((range + 31) & ~31ull, 32), kBfsRange);
			const uint32_t nranges = (uint32_t)((total + range - 1) / range);
			if (nranges > 0)
				bfs_top_down<<<grid_for(nranges, kBfsThreads / 32), kBfsThreads, 0, st>>>(
						out, q, fpos, (uint32_t)qlen, (uint32_t)total, (uint32_t)range, nranges,
						lvl, nq, ctr, cur);
			td_steps++;
			s->launches += 5;
		} else {
			LG_CUDA(cudaMemsetAsync(bits, 0, ((V + 31) / 32) * 4, st), "memset");
			bfs_set_bits<<<grid_for(qlen, 256), 256, 0, st>>>(q, (uint32_t)qlen, bits);
			if (fi)
				bfs_bottom_up_flat<<<grid_for(V, kBfsThreads * kBuVerts), kBfsThreads, 0, st>>>(
						fi->off.as<uint32_t>(), fi->ids.as<uint32_t>(), (uint32_t)V, outdeg,
						bits, lvl, nq, ctr, cur);
			else
				bfs_bottom_up<<<grid_for(V, kBfsThreads), kBfsThreads, 0, st>>>(
						in, outdeg, bits, lvl, nq, ctr, cur);
			bu_steps++;
			s->launches += 2;
		}
		LG_CUDA(cudaGetLastError(), "bfs step");
		LG_TRY(read_words(s, ctr, 2, h));
		qlen = h[0];
		mf = h[1];
		mu -= std::min(mu, (uint64_t)mf);
		reached += qlen;
		reach_edges += mf;
		std::swap(q, nq);
		cur++;
	}
	if (!dev_out) {
		LG_TRY(copy_out(s, levels, lvl, V * 4));
		LG_CUDA(cudaStreamSynchronize(st), "bfs");
	}
	if (result) {
		result->reached = reached;
		result->reach_edges = reach_edges;
		result->max_level = cur - 1;
		result->top_down_steps = td_steps;
		result->bottom_up_steps = bu_steps;
		result->reserved = 0;
	}
	return LG_OK;
}
