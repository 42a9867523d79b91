// lg_sssp.cu - single-source shortest paths with integer edge weights.
//
// Reference: ll_b_sssp_weighted::run (benchmark/benchmarks/sssp.h:97-183), a
// frontier Bellman-Ford to a fixpoint with G_len[e] the per-slot edge
// property (llama/include/llama/ll_mlcsr_properties.h:985-1005); dist[root] =
// 0, unreached vertices keep INT_MAX - 1.  Shortest-path distances are
// unique, so any correct algorithm yields the same array: this one is
// delta-stepping (Meyer & Sanders) in the near/far-queue form.  Vertices
// whose tentative distance is below the current bucket bound are relaxed
// repeatedly from a near queue; improvements beyond the bound go to a far
// pile that is split when the near queue drains, the bound then moving to
// the bucket of the smallest distance left in the pile.  Relaxation is
// atomicMin on 32-bit distances, so the result does not depend on thread
// order.  Per-vertex stamps keep every vertex at most once in the near queue
// of a round and at most once in the far pile, which bounds both by V.
// After lg_snapshot_flatten(snap, 0) the rounds read the flat out-CSR (ids
// and weights in one array each, no deletion bits) instead of the levels.
#include "lg_expand.cuh"
#include "lg_flat.cuh"
#include "lg_sssp.cuh"
#include "lg_sssp_levels.h"
#include "lg_tune.h"

#include <cstring>
#include <new>

namespace lg {

constexpr int kSsspThreads = 256;
constexpr unsigned kRelaxCtasPerSm = 5;
// slots per warp range: LG_TUNE_SSSP_RANGE (1024 by default)

__global__ void sssp_init(uint32_t* dist, uint32_t* stamp, uint32_t* fstamp,
		uint64_t V, uint32_t root, uint32_t* queue) {
	uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (v < V) {
		dist[v] = (v == root) ? 0u : kInf;
		stamp[v] = 0xffffffffu;
		fstamp[v] = 0xffffffffu;
	}
	if (v == 0) queue[0] = root;
}

// One relaxation round over the near queue.  The queue's slot space
// (pos = exclusive prefix of the queued vertices' slot counts, pos[qlen] the
// total, both written earlier on the stream) is cut into `range`-slot
// ranges that the grid's warps take in turn, so a hub in the queue is spread
// over many warps.  ctr[0] near-next length, ctr[1] far length (starts at
// the current pile size), ctr[2] relaxations.
// Registers capped for 5 resident CTAs per SM (48, no spills; 62 uncapped):
// the grid below is exactly the resident CTAs, one wave.
__global__ void __launch_bounds__(kSsspThreads, kRelaxCtasPerSm)
sssp_relax(SnapCsr out, const uint32_t* queue, const uint32_t* pos, uint32_t qlen,
		uint32_t* dist, uint32_t* stamp, uint32_t* fstamp, uint32_t round, uint32_t epoch,
		uint32_t hi, uint32_t* near_next, uint32_t* far, unsigned long long* ctr,
		uint32_t range_max) {
	__shared__ uint32_t sbuf[kSsspThreads / 32][2][kPushBuf];
	const uint32_t lane = threadIdx.x & 31u, wid = threadIdx.x >> 5;
	const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
	unsigned long long relax = sssp_relax_ranges<0>(out, queue, pos, qlen, __ldg(pos + qlen),
			range_max, warp, nwarps, dist, stamp, fstamp, round, epoch, hi, near_next, ctr, far,
			ctr + 1, sbuf[wid][0], sbuf[wid][1]);
	for (int o = 16; o > 0; o >>= 1) relax += __shfl_down_sync(0xffffffffu, relax, o);
	if (lane == 0 && relax) atomicAdd(ctr + 2, relax);
}

// Split the far pile at bound `hi`: entries with lo <= dist < hi go to the
// near queue (entries below lo were settled from a near queue after they
// entered the pile), entries >= hi are kept, stamped with the new epoch, and
// the smallest kept distance is reported in ctr[2].
__global__ void __launch_bounds__(kSsspThreads)
sssp_split_far(const uint32_t* far, unsigned long long n,
		const uint32_t* dist, uint32_t* stamp, uint32_t* fstamp, uint32_t round,
		uint32_t epoch, uint32_t lo, uint32_t hi, uint32_t* near, uint32_t* keep,
		unsigned long long* ctr) {
	__shared__ uint32_t sbuf[kSsspThreads / 32][2][kPushBuf];
	const uint32_t wid = threadIdx.x >> 5;
	unsigned long long m = sssp_split_far_body<0>(far, n, dist, stamp, fstamp, round, epoch,
			lo, hi, near, ctr, keep, ctr + 1, sbuf[wid][0], sbuf[wid][1],
			(uint64_t)blockIdx.x * blockDim.x + threadIdx.x, (uint64_t)gridDim.x * blockDim.x);
	for (int o = 16; o > 0; o >>= 1) m = min(m, __shfl_down_sync(0xffffffffu, m, o));
	if ((threadIdx.x & 31) == 0 && m != ~0ull) atomicMin(ctr + 2, m);
}

// ---------------------------------------------------------------------------
// Light / heavy split.  Edges lighter than delta can improve a vertex inside
// the current bucket, heavier ones only in later buckets, so the rounds of a
// bucket relax only the light edges of the near queue, and each vertex
// settled in the bucket relaxes its heavy edges once when the bucket drains
// (Meyer & Sanders' light/heavy phases).  The flat out-CSR is partitioned per
// row, light edges first (stable), and two one-fragment-per-vertex views
// point at the light and the heavy part of every row.
// ---------------------------------------------------------------------------

// Row v of the flat out-CSR (off, ids, w) rewritten light-first into
// (ids2, w2); lc[v] = its light edges.  A warp per row: a counting pass,
// then a writing pass, 32 edges at a time with ballots (stable).
__global__ void sssp_partition(const uint32_t* off, const uint32_t* ids, const uint32_t* w,
		uint64_t V, uint32_t delta, uint32_t* ids2, uint32_t* w2, uint2* lfr, uint2* hfr) {
	const uint32_t lane = threadIdx.x & 31u;
	const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
	for (uint64_t v = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < V; v += nwarps) {
		const uint32_t b = __ldg(off + v), e = __ldg(off + v + 1);
		uint32_t nl = 0;
		for (uint32_t k = b + lane; k < e + ((32u - (e - b) % 32u) % 32u); k += 32) {
			const bool light = k < e && __ldg(w + k) < delta;
			nl += __popc(__ballot_sync(0xffffffffu, light));
		}
		uint32_t pl = b, ph = b + nl;
		const uint32_t below = (1u << lane) - 1u;
		for (uint32_t k = b + lane; k < e + ((32u - (e - b) % 32u) % 32u); k += 32) {
			const bool in = k < e;
			const uint32_t wk = in ? __ldg(w + k) : 0u;
			const uint32_t ik = in ? __ldg(ids + k) : 0u;
			const bool light = in && wk < delta;
			const unsigned lm = __ballot_sync(0xffffffffu, light);
			const unsigned hm = __ballot_sync(0xffffffffu, in && !light);
			if (light) { const uint32_t d = pl + __popc(lm & below); ids2[d] = ik; w2[d] = wk; }
			else if (in) { const uint32_t d = ph + __popc(hm & below); ids2[d] = ik; w2[d] = wk; }
			pl += __popc(lm);
			ph += __popc(hm);
		}
		if (lane == 0) {
			lfr[v] = make_uint2(b, nl << kLevelBits);
			hfr[v] = make_uint2(b + nl, (e - b - nl) << kLevelBits);
		}
	}
}

__global__ void sssp_iota(uint32_t* a, uint64_t n) {
	const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n) a[i] = (uint32_t)i;
}

// The vertices of the near queue join the bucket's settled list once each
// (stamp = bucket number); ctr[3] counts the list.
__global__ void sssp_collect(const uint32_t* q, uint32_t n, uint32_t* bstamp, uint32_t bucket,
		uint32_t* blist, unsigned long long* ctr) {
	__shared__ uint32_t sbuf[kSsspThreads / 32][kPushBuf];
	sssp_collect_body<0>(q, n, bstamp, bucket, blist, ctr + 3, sbuf[threadIdx.x >> 5],
			(uint64_t)blockIdx.x * blockDim.x + threadIdx.x, (uint64_t)gridDim.x * blockDim.x);
}

__global__ void sssp_reach(const uint32_t* dist, const uint32_t* outdeg, uint64_t V,
		unsigned long long* ctr) {
	unsigned long long c = 0, e = 0, mx = 0;
	for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < V;
			v += (uint64_t)gridDim.x * blockDim.x) {
		uint32_t d = dist[v];
		if (d < kInf) { c++; e += outdeg[v]; if (d > mx) mx = d; }
	}
	for (int o = 16; o > 0; o >>= 1) {
		c += __shfl_down_sync(0xffffffffu, c, o);
		e += __shfl_down_sync(0xffffffffu, e, o);
		mx = max(mx, __shfl_down_sync(0xffffffffu, mx, o));
	}
	if ((threadIdx.x & 31) == 0) {
		atomicAdd(ctr, c);
		atomicAdd(ctr + 1, e);
		atomicMax(ctr + 2, mx);
	}
}

} // namespace lg

using namespace lg;

struct lg_sssp_split {
	uint32_t delta = 0;
	DevBuf ids, w;          // E: the flat out-CSR, each row light edges first
	DevBuf lfr, hfr;        // V: one fragment per row, light part / heavy part
	DevBuf fidx;            // V + 1: fragment index of every row (the identity)
	DevBuf zeros;           // deletion bitset of the view (none deleted)
	DevBuf lt_light, lt_heavy;   // device LevelTabs of the two views
	SnapCsr view(bool heavy, const uint32_t* deg, uint64_t V) const {
		SnapCsr c;
		c.frag_off = fidx.as<uint32_t>();
		c.frags = (heavy ? hfr : lfr).as<uint2>();
		c.lt = (heavy ? lt_heavy : lt_light).as<LevelTab>();
		c.deg = deg;
		c.V = V;
		return c;
	}
};

void lg_free_sssp_split(lg_sssp_split* p) { delete p; }

namespace {

// The snapshot's out-CSR flattened (the snapshot's own flat CSR when it has
// one with weights, else one built here and dropped after) and split for
// `delta`; kept on the snapshot for the next call with the same delta.
lg_status ensure_split(lg_snapshot* sn, uint32_t delta) {
	if (sn->sssp_split && sn->sssp_split->delta == delta) return LG_OK;
	lg_store* s = sn->store;
	cudaStream_t st = s->stream;
	const uint64_t V = sn->V;
	lg_sssp_split* p = sn->sssp_split;
	if (!p) {
		p = new (std::nothrow) lg_sssp_split();
		if (!p) return set_error(LG_ENOMEM, "host allocation");
		sn->sssp_split = p;
	}
	p->delta = 0;
	FlatCsr own;
	const FlatCsr* f = sn->flat[0];
	if (!f || !f->weighted) {
		LG_TRY(build_flat(sn, 0, own, false));
		if (!own.weighted) return set_error(LG_ESTATE, "the out-CSR carries no edge weights");
		f = &own;
	}
	const uint64_t E = f->E;
	LG_TRY(p->ids.reserve(std::max<uint64_t>(E, 1) * 4));
	LG_TRY(p->w.reserve(std::max<uint64_t>(E, 1) * 4));
	LG_TRY(p->lfr.reserve(std::max<uint64_t>(V, 1) * sizeof(uint2)));
	LG_TRY(p->hfr.reserve(std::max<uint64_t>(V, 1) * sizeof(uint2)));
	LG_TRY(p->fidx.reserve((V + 1) * 4));
	const uint64_t words = E / 32 + 2;
	LG_TRY(p->zeros.reserve(words * 4));
	LG_TRY(p->lt_light.reserve(sizeof(LevelTab)));
	LG_TRY(p->lt_heavy.reserve(sizeof(LevelTab)));
	LG_CUDA(cudaMemsetAsync(p->zeros.p, 0, words * 4, st), "memset");
	int sms = 148;
	cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->device);
	sssp_partition<<<(unsigned)sms * 16u, 256, 0, st>>>(f->off.as<uint32_t>(),
			f->ids.as<uint32_t>(), f->w.as<uint32_t>(), V, delta, p->ids.as<uint32_t>(),
			p->w.as<uint32_t>(), p->lfr.as<uint2>(), p->hfr.as<uint2>());
	sssp_iota<<<grid_for(V + 1, 256), 256, 0, st>>>(p->fidx.as<uint32_t>(), V + 1);
	LG_CUDA(cudaGetLastError(), "sssp_partition");
	s->launches += 2;
	LevelTab lt;
	memset(&lt, 0, sizeof(lt));
	lt.ids[0] = p->ids.as<uint32_t>();
	lt.w[0] = p->w.as<uint32_t>();
	lt.del[0] = p->zeros.as<uint32_t>();
	LG_CUDA(cudaMemcpyAsync(p->lt_light.p, &lt, sizeof(lt), cudaMemcpyHostToDevice, st), "h2d");
	LG_CUDA(cudaMemcpyAsync(p->lt_heavy.p, &lt, sizeof(lt), cudaMemcpyHostToDevice, st), "h2d");
	LG_CUDA(cudaStreamSynchronize(st), "sssp split");    // `own` and `lt` go out of scope
	s->h2d_bytes += 2 * sizeof(lt);
	p->delta = delta;
	return LG_OK;
}

} // namespace

extern "C" lg_status lg_sssp_delta(lg_snapshot* sn, int64_t root, uint32_t delta,
		uint32_t* dist, lg_sssp_result* result) {
	clear_error();
	if (!sn || !dist) return set_error(LG_EINVAL, "null argument");
	if (root < 0 || (uint64_t)root >= sn->V)
		return set_error(LG_EINVAL, "root %lld out of range", (long long)root);
	if (delta == 0) return set_error(LG_EINVAL, "delta must be positive");
	lg_store* s = sn->store;
	for (int l = sn->min_level; l <= sn->level; l++)
		if (!s->out.levels[l]->w.p && s->out.levels[l]->n_fragment_slots > 0)
			return set_error(LG_ESTATE, "level %d of the out-CSR carries no edge weights", l);
	LG_CUDA(cudaSetDevice(s->device), "cudaSetDevice");
	cudaStream_t st = s->stream;
	const uint64_t V = sn->V;
	DevBuf* sc = s->scratch;
	LG_TRY(sc[0].reserve(V * 4));          // near queue
	LG_TRY(sc[1].reserve(V * 4));          // next near queue
	LG_TRY(sc[2].reserve(V * 4));          // far pile
	LG_TRY(sc[3].reserve(V * 4));          // far pile being compacted
	LG_TRY(sc[5].reserve(2 * V * 4));      // near and far stamps
	LG_TRY(sc[6].reserve(8 * sizeof(unsigned long long)));     // counters (4 used)
	LG_TRY(sc[7].reserve((2 * V + 1) * 4));   // queue slot counts and their prefix
	uint32_t* qcnt = sc[7].as<uint32_t>();
	uint32_t* qpos = qcnt + V;
	int sms = 148;
	cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->device);
	const unsigned relax_blocks = (unsigned)sms * kRelaxCtasPerSm;   // persistent, one wave
	const uint32_t range = (uint32_t)tune_value(s->device, LG_TUNE_SSSP_RANGE);
	const bool dev_out = is_device_pointer(dist);
	uint32_t* d = dist;
	if (!dev_out) { LG_TRY(sc[4].reserve(V * 4)); d = sc[4].as<uint32_t>(); }
	uint32_t* q = sc[0].as<uint32_t>();
	uint32_t* qn = sc[1].as<uint32_t>();
	uint32_t* far = sc[2].as<uint32_t>();
	uint32_t* far2 = sc[3].as<uint32_t>();
	uint32_t* stamp = sc[5].as<uint32_t>();
	uint32_t* fstamp = stamp + V;
	unsigned long long* ctr = sc[6].as<unsigned long long>();
	// the one-fragment view of a flattened out-CSR when there is one
	const FlatCsr* fo = sn->flat[0];
	SnapCsr out = (fo && fo->has_view && fo->weighted)
			? fo->view(sn->out.deg.as<uint32_t>()) : sn->view(0);
	// light / heavy split (LG_TUNE_SSSP_SPLIT): rounds walk the light view,
	// the bucket's settled list walks the heavy view once
	const bool split = tune_value(s->device, LG_TUNE_SSSP_SPLIT) != 0;
	SnapCsr heavy = out;
	uint32_t* blist = nullptr;
	uint32_t* bstamp = nullptr;
	if (split) {
		LG_TRY(ensure_split(sn, delta));
		out = sn->sssp_split->view(false, sn->out.deg.as<uint32_t>(), V);
		heavy = sn->sssp_split->view(true, sn->out.deg.as<uint32_t>(), V);
		LG_TRY(sc[9].reserve(V * 4));
		LG_TRY(sc[10].reserve(V * 4));
		blist = sc[9].as<uint32_t>();
		bstamp = sc[10].as<uint32_t>();
		LG_CUDA(cudaMemsetAsync(bstamp, 0xff, V * 4, st), "memset");
	}

	sssp_init<<<grid_for(V, 256), 256, 0, st>>>(d, stamp, fstamp, V, (uint32_t)root, q);
	LG_CUDA(cudaGetLastError(), "sssp_init");
	s->launches++;
	uint64_t qlen = 1, flen = 0, blen = 0, relaxations = 0;
	uint32_t hi = delta, round = 0, epoch = 0, bid = 0;
	int buckets = 1;
	// counters read back and round set-ups written through the store's
	// pinned words (no pageable staging on every round)
	unsigned long long* hw = nullptr;
	LG_TRY(host_words(s, &hw));
	unsigned long long* h = hw;              // 4 words read back
	unsigned long long* init = hw + 4;       // 4 words written
	LG_CUDA(cudaMemsetAsync(ctr, 0, 4 * sizeof(unsigned long long), st), "memset");
	// the same rounds in one cooperative launch (LG_TUNE_SSSP_LEVELS)
	bool one_launch = false;
	if (tune_value(s->device, LG_TUNE_SSSP_LEVELS)) {
		SsspLevelsArgs a;
		a.out = out;
		a.heavy = heavy;
		a.split = split ? 1 : 0;
		a.q = q; a.qn = qn; a.far = far; a.far2 = far2;
		a.dist = d; a.stamp = stamp; a.fstamp = fstamp; a.bstamp = bstamp; a.blist = blist;
		a.cnt = qcnt; a.pos = qpos;
		a.bsum = nullptr;
		a.V = V;
		a.delta = delta;
		a.range_max = range;
		int r = 0, b = 0;
		uint64_t rx = 0;
		LG_TRY(sssp_levels_run(s, a, sc[11], &r, &b, &rx, &one_launch));
		if (one_launch) {
			round = (uint32_t)r;
			buckets = b;
			relaxations = rx;
			qlen = flen = blen = 0;
		}
	}
	while (qlen > 0 || flen > 0 || blen > 0) {
		if (qlen == 0 && blen > 0) {
			// the bucket has drained: its settled vertices relax their
			// heavy edges once (every such relaxation lands at >= hi, in
			// the far pile)
			round++;
			init[0] = 0; init[1] = flen; init[2] = 0; init[3] = 0;
			LG_CUDA(cudaMemcpyAsync(ctr, init, 4 * sizeof(unsigned long long),
					cudaMemcpyHostToDevice, st), "h2d");
			s->h2d_bytes += 4 * sizeof(unsigned long long);
			list_slots<<<grid_for(blen, 256), 256, 0, st>>>(heavy, blist, (uint32_t)blen, qcnt);
			LG_TRY(exclusive_scan_u32(qcnt, qpos, blen, sc[8], st, nullptr));
			sssp_relax<<<relax_blocks, kSsspThreads, 0, st>>>(heavy, blist, qpos, (uint32_t)blen,
					d, stamp, fstamp, round, epoch, hi, qn, far, ctr, range);
			LG_CUDA(cudaGetLastError(), "sssp_relax heavy");
			s->launches += 5;
			LG_CUDA(cudaMemcpyAsync(h, ctr, 4 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st), "d2h");
			LG_CUDA(cudaStreamSynchronize(st), "sssp heavy");
			s->d2h_bytes += 4 * sizeof(unsigned long long);
			if (h[0] != 0 || h[1] > V) return set_error(LG_ECUDA, "sssp heavy phase out of bounds");
			flen = h[1];
			relaxations += h[2];
			blen = 0;
			bid++;
			continue;
		}
		if (qlen == 0) {
			// near queue drained: split the far pile at the next bound; if
			// nothing falls below it, jump to the bucket of the smallest
			// remaining distance and split again
			uint32_t lo = hi;
			hi = (hi > kInf - delta) ? kInf : hi + delta;
			for (int attempt = 0; attempt < 2; attempt++) {
				round++;
				epoch++;
				init[0] = 0; init[1] = 0; init[2] = ~0ull; init[3] = 0;
				LG_CUDA(cudaMemcpyAsync(ctr, init, 4 * sizeof(unsigned long long),
						cudaMemcpyHostToDevice, st), "h2d");
				s->h2d_bytes += 4 * sizeof(unsigned long long);
				const unsigned split_blocks = (unsigned)std::min<uint64_t>(
						std::max<uint64_t>(grid_for(flen, kSsspThreads), 1), relax_blocks);
				sssp_split_far<<<split_blocks, kSsspThreads, 0, st>>>(far, flen, d, stamp,
						fstamp, round, epoch, lo, hi, q, far2, ctr);
				LG_CUDA(cudaGetLastError(), "sssp_split_far");
				s->launches++;
				LG_CUDA(cudaMemcpyAsync(h, ctr, 3 * sizeof(unsigned long long),
						cudaMemcpyDeviceToHost, st), "d2h");
				LG_CUDA(cudaStreamSynchronize(st), "sssp split");
				s->d2h_bytes += 4 * sizeof(unsigned long long);
				if (h[0] > V || h[1] > V) return set_error(LG_ECUDA, "sssp queue overflow");
				qlen = h[0];
				flen = h[1];
				std::swap(far, far2);
				buckets++;
				if (qlen > 0 || flen == 0) break;
				uint32_t mind = (uint32_t)h[2];
				lo = (mind / delta) * delta;
				hi = (lo > kInf - delta) ? kInf : lo + delta;
			}
			continue;
		}
		round++;
		init[0] = 0; init[1] = flen; init[2] = 0; init[3] = blen;
		LG_CUDA(cudaMemcpyAsync(ctr, init, 4 * sizeof(unsigned long long),
				cudaMemcpyHostToDevice, st), "h2d");
		s->h2d_bytes += 4 * sizeof(unsigned long long);
		if (split) {
			sssp_collect<<<(unsigned)std::min<uint64_t>(grid_for(qlen, kSsspThreads), relax_blocks),
					kSsspThreads, 0, st>>>(q, (uint32_t)qlen, bstamp, bid, blist, ctr);
			s->launches++;
		}
		list_slots<<<grid_for(qlen, 256), 256, 0, st>>>(out, q, (uint32_t)qlen, qcnt);
		LG_TRY(exclusive_scan_u32(qcnt, qpos, qlen, sc[8], st, nullptr));
		sssp_relax<<<relax_blocks, kSsspThreads, 0, st>>>(out, q, qpos, (uint32_t)qlen, d,
				stamp, fstamp, round, epoch, hi, qn, far, ctr, range);
		LG_CUDA(cudaGetLastError(), "sssp_relax");
		s->launches += 5;
		LG_CUDA(cudaMemcpyAsync(h, ctr, 4 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st), "d2h");
		LG_CUDA(cudaStreamSynchronize(st), "sssp relax");
		s->d2h_bytes += 4 * sizeof(unsigned long long);
		if (h[0] > V || h[1] > V) return set_error(LG_ECUDA, "sssp queue overflow");
		qlen = h[0];
		flen = h[1];
		relaxations += h[2];
		if (split) blen = h[3];
		if (blen > V) return set_error(LG_ECUDA, "sssp settled list overflow");
		std::swap(q, qn);
	}
	LG_CUDA(cudaMemsetAsync(ctr, 0, 3 * sizeof(unsigned long long), st), "memset");
	sssp_reach<<<592, 256, 0, st>>>(d, sn->out.deg.as<uint32_t>(), V, ctr);
	LG_CUDA(cudaGetLastError(), "sssp_reach");
	s->launches++;
	LG_CUDA(cudaMemcpyAsync(h, ctr, 4 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st), "d2h");
	s->d2h_bytes += 4 * sizeof(unsigned long long);
	if (!dev_out) LG_TRY(copy_out(s, dist, d, V * 4));
	LG_CUDA(cudaStreamSynchronize(st), "sssp");
	if (result) {
		result->reached = h[0];
		result->reach_edges = h[1];
		result->max_dist = (uint32_t)h[2];
		result->buckets = buckets;
		result->rounds = (int32_t)round;
		result->relaxations = relaxations;
	}
	return LG_OK;
}
