// lg_flat.cu - flattening a snapshot direction into one CSR on the device.
//
// Reference: ll_t_flatten (benchmark/tools/flatten.h) merges every level of
// a LLAMA graph into a single level by iterating each vertex's edges
// (newest fragment first, deleted edges skipped) on the host.  Here the
// same order is produced in one balanced pass over the virtual slot space
// (one CTA per 1024 virtual slots): row starts are the scan of the live
// degrees, and flat_write writes every live slot's id (and weight) at its
// block's base (found from the row start of the block's first vertex) + its
// live rank.  Row bookkeeping for the tile kernels (heads, nz_rows,
// nz_off, tile_seg) and the optional fragment view follow.
#include "lg_flat.cuh"

#include <algorithm>
#include <cstring>

namespace lg {

// Writes the live slots of block r to ids[base ...] in slot order (and their
// weights to w when non-null).  base = the live slots before the block:
// off[e] of the entry e that holds the block's first slot, plus e's live
// slots before it (its deleted slots counted a word at a time).  off is the
// exclusive scan of the snapshot's live degrees; every entry that starts in
// the block checks it against its rank in the block, and a mismatch (a
// degree that is not the live slot count) sets bit 2 of *err.
__global__ void __launch_bounds__(kMapThreads)
flat_write(SlotSpace sp, const uint32_t* off, uint32_t E, uint32_t* ids, uint32_t* w,
		unsigned int* err) {
	constexpr int kGroups = kMapPerThread * (kMapThreads / 32);
	__shared__ BlockMap m;
	__shared__ uint16_t rank[kMapRange];
	__shared__ uint32_t gpre[kGroups];
	__shared__ uint32_t dead_w[kMapThreads / 32];
	const uint32_t tid = threadIdx.x, lane = tid & 31u, wid = tid >> 5;
	const uint32_t r = blockIdx.x, ra = r * kMapRange, rb = block_end(sp, r);
	map_block(sp, r, ra, rb, m);

	// the block's slots: deletion word, id (and weight) loads issued first,
	// for every slot, so they overlap the count below
	uint32_t dw[kMapPerThread], id[kMapPerThread], wt[kMapPerThread], mask[kMapPerThread];
	uint32_t bit[kMapPerThread];
	bool have[kMapPerThread];
#pragma unroll
	for (int u = 0; u < kMapPerThread; u++) {
		uint32_t lv = 0, idx = 0;
		have[u] = block_slot(m, ra, rb, u * kMapThreads + tid, &lv, &idx);
		dw[u] = have[u] ? __ldg(sp.g.lt->del[lv] + (idx >> 5)) : 0u;
		id[u] = have[u] ? __ldg(sp.g.lt->ids[lv] + idx) : 0u;
		wt[u] = (have[u] && w) ? __ldg(sp.g.lt->w[lv] + idx) : 0u;
		bit[u] = idx & 31u;
	}

	// the first entry's slots before ra: its fragments lead ftab
	const uint32_t e0 = m.eb;
	uint32_t before = 0, dead = 0;
	if (m.nf > 0 && m.fstart[0] < ra) {
		const uint32_t nfe = min(__ldg(sp.g.frag_off + e0 + 1) - __ldg(sp.g.frag_off + e0), m.nf);
		for (uint32_t i = 0; i < nfe; i++) {
			const uint32_t s0 = m.fstart[i];
			if (s0 >= ra) break;
			const uint2 fr = m.ftab[i];
			const uint32_t n = min(frag_len(fr), ra - s0);
			before += n;
			const uint32_t* d = sp.g.lt->del[frag_level(fr)];
			const uint32_t a = fr.x, b = fr.x + n;          // slots [a, b)
			for (uint32_t wd = (a >> 5) + tid; wd <= ((b - 1) >> 5); wd += kMapThreads) {
				uint32_t x = __ldg(d + wd);
				if (wd == (a >> 5)) x &= ~0u << (a & 31);
				if (wd == ((b - 1) >> 5) && (b & 31)) x &= (1u << (b & 31)) - 1u;
				dead += __popc(x);
			}
		}
	}
#pragma unroll
	for (int o = 16; o > 0; o >>= 1) dead += __shfl_xor_sync(0xffffffffu, dead, o);
	if (lane == 0) dead_w[wid] = dead;

#pragma unroll
	for (int u = 0; u < kMapPerThread; u++)
		mask[u] = __ballot_sync(0xffffffffu, have[u] && !((dw[u] >> bit[u]) & 1u));
	// slot order is k = u * kMapThreads + wid * 32 + lane: group u * 4 + wid
	if (lane == 0) {
#pragma unroll
		for (int u = 0; u < kMapPerThread; u++)
			gpre[u * (kMapThreads / 32) + wid] = __popc(mask[u]);
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
	uint32_t dead_all = 0;
#pragma unroll
	for (int x = 0; x < kMapThreads / 32; x++) dead_all += dead_w[x];
	const uint32_t base = __ldg(off + e0) + before - dead_all;
	const uint32_t below = (1u << lane) - 1u;
#pragma unroll
	for (int u = 0; u < kMapPerThread; u++) {
		const uint32_t k = u * kMapThreads + tid;
		const uint32_t rk = gpre[u * (kMapThreads / 32) + wid] + __popc(mask[u] & below);
		rank[k] = (uint16_t)rk;
		if ((mask[u] >> lane) & 1u) {
			if (base + rk < E) {
				ids[base + rk] = id[u];
				if (w) w[base + rk] = wt[u];
			} else {
				atomicOr(err, 2u);      // degrees and live slots disagree
			}
		}
	}
	__syncthreads();
	// entries starting in the block: their row start must be base + rank
	const uint32_t e_begin = __ldg(sp.range_lb + r);
	const uint32_t e_end = r == sp.nranges - 1 ? (uint32_t)sp.g.V : __ldg(sp.range_lb + r + 1);
	bool bad = false;
	for (uint32_t e = e_begin + tid; e < e_end; e += kMapThreads) {
		const uint32_t p = __ldg(sp.pos + e);
		if (p < rb && p >= ra) bad |= __ldg(off + e) != base + rank[p - ra];
	}
	if (r == sp.nranges - 1 && tid == kMapThreads - 1) {
		// the last block ends at the total of the degrees
		const uint32_t nlive = gpre[kGroups - 1] + __popc(mask[kMapPerThread - 1]);
		bad |= base + nlive != __ldg(off + sp.g.V);
	}
	if (bad) atomicOr(err, 2u);
}

__global__ void flat_flags(const uint32_t* off, uint64_t V, uint32_t* flags) {
	const uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (v >= V) return;
	flags[v] = __ldg(off + v + 1) > __ldg(off + v);
}

__global__ void flat_rows(const uint32_t* off, const uint32_t* kidx, uint64_t V,
		uint32_t* nz_rows, uint32_t* nz_off, uint32_t* heads) {
	const uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (v >= V) return;
	const uint32_t o = __ldg(off + v);
	if (__ldg(off + v + 1) == o) return;
	const uint32_t k = __ldg(kidx + v);
	nz_rows[k] = (uint32_t)v;
	nz_off[k] = o;
	atomicOr(heads + (o >> 5), 1u << (o & 31u));
}

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

// Fragment view: row k of the flat CSR is fragment k, {start, len << 6 | 0};
// a row longer than a fragment can describe sets *err.
__global__ void flat_view(const uint32_t* nz_off, uint32_t R, uint32_t E,
		uint2* frags, unsigned int* err) {
	const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
	if (k >= R) return;
	const uint32_t st = __ldg(nz_off + k);
	const uint32_t en = k + 1 < R ? __ldg(nz_off + k + 1) : E;
	const uint32_t len = en - st;
	if (len > (uint32_t)LG_MAX_FRAGMENT_LEN) { atomicOr(err, 1u); return; }
	frags[k] = make_uint2(st, len << kLevelBits);
}

SlotSpace slot_space(const lg_snapshot* sn, int dir) {
	const SnapDir& d = dir == 0 ? sn->out : sn->in;
	SlotSpace sp;
	sp.g = sn->view(dir);
	sp.pos = d.slot_off.as<uint32_t>();
	sp.range_lb = d.range_lb.as<uint32_t>();
	sp.total = (uint32_t)d.n_frag_slots;
	sp.nranges = (uint32_t)std::max<uint64_t>(1, (sp.total + kMapRange - 1) / kMapRange);
	return sp;
}

lg_status build_flat(lg_snapshot* sn, int dir, FlatCsr& f, bool view) {
	lg_store* s = sn->store;
	cudaStream_t st = s->stream;
	const SlotSpace sp = slot_space(sn, dir);
	const uint64_t V = sn->V;
	const unsigned B = 256;
	const DevCsr& csr = dir == 0 ? s->out : s->in;
	// edge weights are read only along out-edges (SSSP), so only the out
	// direction carries them into the flat CSR
	bool weighted = dir == 0;
	for (int l = sn->min_level; l <= sn->level && weighted; l++)
		if (csr.levels[l]->n_fragment_slots > 0 && !csr.levels[l]->w.p) weighted = false;

	f.V = V;
	f.has_view = false;
	f.has_nz_outdeg = false;
	// row starts from the live degrees; flat_write checks them
	const SnapDir& d = dir == 0 ? sn->out : sn->in;
	const uint64_t E = d.n_edges;
	if (E > 0xffffffffull - 2 * kFlatTile)
		return set_error(LG_ENOTSUP, "more than 2^32 - %u live edges in one direction",
				2 * kFlatTile);
	f.E = E;
	f.weighted = weighted;
	f.ntiles = (uint32_t)((E + kFlatTile - 1) / kFlatTile);
	LG_TRY(f.ids.reserve(std::max<uint64_t>(E, 1) * sizeof(uint32_t)));
	if (weighted) LG_TRY(f.w.reserve(std::max<uint64_t>(E, 1) * sizeof(uint32_t)));
	LG_TRY(f.off.reserve((V + 1) * sizeof(uint32_t)));
	LG_TRY(f.kidx.reserve((V + 1) * sizeof(uint32_t)));
	LG_TRY(f.err.reserve(sizeof(unsigned int)));
	uint32_t* off = f.off.as<uint32_t>();
	LG_CUDA(cudaMemsetAsync(f.err.p, 0, sizeof(unsigned int), st), "clear flag");
	LG_TRY(exclusive_scan_u32(d.deg.as<uint32_t>(), off, V, f.scan_tmp, st, nullptr));
	flat_write<<<sp.nranges, kMapThreads, 0, st>>>(sp, off, (uint32_t)E, f.ids.as<uint32_t>(),
			weighted ? f.w.as<uint32_t>() : nullptr, f.err.as<unsigned int>());
	LG_CUDA(cudaGetLastError(), "flat_write");
	unsigned int err = 0;
	LG_CUDA(cudaMemcpyAsync(&err, f.err.p, sizeof(err), cudaMemcpyDeviceToHost, st), "d2h");
	LG_TRY(f.flags.reserve(std::max<uint64_t>(V, 1) * sizeof(uint32_t)));
	flat_flags<<<grid_for(V, B), B, 0, st>>>(off, V, f.flags.as<uint32_t>());
	LG_CUDA(cudaGetLastError(), "flat_flags");
	uint64_t R = 0;
	LG_TRY(exclusive_scan_u32(f.flags.as<uint32_t>(), f.kidx.as<uint32_t>(), V, f.scan_tmp,
			st, &R));
	// (the scan waited for the stream, so err is in)
	if (err & 2u)
		return set_error(LG_EINVAL, "a vertex's degree differs from its live edge count");
	f.R = R;
	const uint64_t head_words = (uint64_t)f.ntiles * kFlatTileWords + 1;
	LG_TRY(f.rows.reserve((2 * f.rcap() + f.ntiles + head_words) * sizeof(uint32_t)));
	uint32_t* heads = const_cast<uint32_t*>(f.heads());
	LG_CUDA(cudaMemsetAsync(heads, 0, head_words * sizeof(uint32_t), st), "clear heads");
	flat_rows<<<grid_for(V, B), B, 0, st>>>(off, f.kidx.as<uint32_t>(), V,
			const_cast<uint32_t*>(f.nz_rows()), const_cast<uint32_t*>(f.nz_off()), heads);
	LG_CUDA(cudaGetLastError(), "flat_rows");
	if (f.ntiles > 0) {
		flat_tiles<<<grid_for(f.ntiles, B), B, 0, st>>>(f.nz_off(), (uint32_t)R, f.ntiles,
				const_cast<uint32_t*>(f.tile_seg()));
		LG_CUDA(cudaGetLastError(), "flat_tiles");
	}
	s->launches += 3 + 1 + 1 + 3 + 1 + (f.ntiles > 0);
	if (!view) return LG_OK;

	LG_TRY(f.vfrags.reserve(f.rcap() * sizeof(uint2)));
	const uint64_t del_words = (E + 31) / 32 + 1;
	LG_TRY(f.vdel.reserve(del_words * sizeof(uint32_t)));
	LG_CUDA(cudaMemsetAsync(f.vdel.p, 0, del_words * sizeof(uint32_t), st), "clear view bits");
	LG_CUDA(cudaMemsetAsync(f.err.p, 0, sizeof(unsigned int), st), "clear flag");
	if (R > 0) {
		flat_view<<<grid_for(R, B), B, 0, st>>>(f.nz_off(), (uint32_t)R, (uint32_t)E,
				f.vfrags.as<uint2>(), f.err.as<unsigned int>());
		LG_CUDA(cudaGetLastError(), "flat_view");
		s->launches++;
	}
	LevelTab lt;
	std::memset(&lt, 0, sizeof(lt));
	lt.ids[0] = f.ids.as<uint32_t>();
	lt.del[0] = f.vdel.as<uint32_t>();
	lt.w[0] = weighted ? f.w.as<uint32_t>() : nullptr;
	LG_TRY(f.vlt.reserve(sizeof(LevelTab)));
	LG_CUDA(cudaMemcpyAsync(f.vlt.p, &lt, sizeof(lt), cudaMemcpyHostToDevice, st), "level table");
	LG_CUDA(cudaMemcpyAsync(&err, f.err.p, sizeof(err), cudaMemcpyDeviceToHost, st), "d2h");
	LG_CUDA(cudaStreamSynchronize(st), "flatten");
	if (err)
		return set_error(LG_ENOTSUP, "a vertex has more than %u live edges, the longest "
				"fragment a flat view can describe", (unsigned)LG_MAX_FRAGMENT_LEN);
	f.has_view = true;
	return LG_OK;
}

} // namespace lg

using namespace lg;

extern "C" lg_status lg_snapshot_flatten(lg_snapshot* sn, int dir) {
	clear_error();
	if (!sn) return set_error(LG_EINVAL, "null argument");
	if (dir != 0 && dir != 1) return set_error(LG_EINVAL, "dir must be 0 or 1");
	const SnapDir& d = dir == 0 ? sn->out : sn->in;
	if (!d.present) return set_error(LG_ESTATE, "the store has no in-CSR");
	if (sn->flat[dir]) return LG_OK;
	lg_store* s = sn->store;
	LG_CUDA(cudaSetDevice(s->device), "cudaSetDevice");
	// reuse the device memory of a flat CSR an earlier snapshot released
	FlatCsr* f = nullptr;
	for (int i = 0; i < 2 && !f; i++)
		if (s->flat_spare[i]) { f = s->flat_spare[i]; s->flat_spare[i] = nullptr; }
	if (!f) f = new FlatCsr;
	// the fragment view is read by the out-direction traversals only
	const lg_status st = build_flat(sn, dir, *f, dir == 0);
	if (st != LG_OK) {
		cudaStreamSynchronize(s->stream);
		delete f;
		return st;
	}
	sn->flat[dir] = f;
	return LG_OK;
}

void lg_flat_release(lg_store* s, FlatCsr* f) {
	if (!f) return;
	for (int i = 0; i < 2; i++)
		if (!s->flat_spare[i]) { s->flat_spare[i] = f; return; }
	delete f;
}

extern "C" lg_status lg_snapshot_unflatten(lg_snapshot* sn) {
	clear_error();
	if (!sn) return set_error(LG_EINVAL, "null argument");
	LG_CUDA(cudaSetDevice(sn->store->device), "cudaSetDevice");
	LG_CUDA(cudaStreamSynchronize(sn->store->stream), "unflatten");
	for (int d = 0; d < 2; d++) {
		lg_flat_release(sn->store, sn->flat[d]);
		sn->flat[d] = nullptr;
	}
	return LG_OK;
}

extern "C" lg_status lg_snapshot_is_flat(const lg_snapshot* sn, int dir, int* flat) {
	if (!sn || !flat) return set_error(LG_EINVAL, "null argument");
	if (dir != 0 && dir != 1) return set_error(LG_EINVAL, "dir must be 0 or 1");
	*flat = sn->flat[dir] != nullptr;
	return LG_OK;
}
