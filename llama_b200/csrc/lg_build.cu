// lg_build.cu - building the next level of a store on the device from an
// edge delta.
//
// Reference: a LLAMA level is written by ll_mlcsr_core::init_level_from_degrees
// / init_node / write_values / finish_level_vertices
// (llama/include/llama/ll_mlcsr_sp.h:1375-1715), the in-CSR by
// make_reverse_edges (llama/include/llama/ll_mlcsr_graph.h:955-1058), and
// deletions lower the max_visible_level of the deleted edge's slot in an
// older level (ll_writable_graph.h:936-945).  lg_store_build_level produces
// the same vertex tables and edge slots on the device (the layout a level
// built that way on the host and passed to lg_store_ingest_level has), from
// the new edges and the deleted edges alone:
//
//   1. new edges as (src << 32 | dst) keys, radix sorted (weights follow);
//      ids in range, no duplicates;
//   2. deleted edges sorted the same way and located in the previous
//      snapshot by walking the vertex's fragment chain (binary search in each
//      sorted fragment, skipping slots deleted at or before it); a new edge
//      must not be live there already;
//   3. per vertex, the element init_node gives it (bl_node: length, degree,
//      continuation record) and the slots it takes; a scan places the
//      fragments in vertex order and bl_fill writes every new edge's id (and
//      weight) into its slot; continuation records and unused slots hold
//      0xffffffff as in an ingested level;
//   4. the in-CSR the same way from (dst << 32 | src) keys;
//   5. every deletion becomes a mark (slot index, slot level << 26 | new
//      level) in the store's deletion list.
// Everything is checked before anything is committed: on an error the store
// is left as it was.
#include "lg_device.cuh"
#include "lg_sort.cuh"

#include <algorithm>
#include <cstring>
#include <vector>

namespace lg {

// Device view of the levels already in one direction of the store, with the
// deletion bitsets of the snapshot the new level builds on.
struct BuildTab {
	const lg_vt_entry* vt[LG_MAX_LEVELS];
	const uint32_t* ids[LG_MAX_LEVELS];
	const uint32_t* del[LG_MAX_LEVELS];
	uint64_t max_nodes[LG_MAX_LEVELS];
	int min_level;             // levels below are aged out (null above)
};

enum BuildErr : unsigned {
	kErrRange = 1u, kErrDupNew = 2u, kErrDupDel = 4u, kErrNotLive = 8u, kErrLive = 16u,
};

__global__ void bl_keys(const uint32_t* a, const uint32_t* b, uint64_t n, uint64_t V,
		unsigned long long* keys, uint32_t* idx, unsigned* err) {
	const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	const uint32_t x = a[i], y = b[i];
	if (x >= V || y >= V) atomicOr(err, kErrRange);
	keys[i] = ((unsigned long long)x << 32) | y;
	if (idx) idx[i] = (uint32_t)i;
}

// (hi, lo) -> (lo, hi) of sorted keys
__global__ void bl_swap(const unsigned long long* k, uint64_t n, unsigned long long* out) {
	const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	const unsigned long long x = k[i];
	out[i] = (x << 32) | (x >> 32);
}

__global__ void bl_dups(const unsigned long long* k, uint64_t n, unsigned* err, unsigned bit) {
	const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i == 0 || i >= n) return;
	if (k[i] == k[i - 1]) atomicOr(err, bit);
}

__global__ void bl_count(const unsigned long long* k, uint64_t n, uint32_t* cnt) {
	const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	atomicAdd(cnt + (uint32_t)(k[i] >> 32), 1u);
}

__global__ void bl_mark(const uint2* dels, uint64_t n, int L, BuildTab t) {
	const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	const uint2 d = dels[i];
	const uint32_t lv = d.y >> LG_BITS_LEVEL;
	const uint32_t ml = d.y & ((1u << LG_BITS_LEVEL) - 1u);
	if ((int)lv > L || (int)lv < t.min_level || (int)ml > L) return;
	atomicOr(const_cast<uint32_t*>(t.del[lv]) + (d.x >> 5), 1u << (d.x & 31));
}

// Edge id of the slot holding (v -> x) live in snapshot `snap`, or -1: the
// walk of iter_begin / iter_descend (ll_mlcsr_sp.h:1994-2134), each
// fragment binary searched (fragments are sorted by neighbour id), ending at
// the aged-out levels.
__device__ int64_t find_live(const BuildTab& t, int snap, uint32_t v, uint32_t x) {
	if (v >= t.max_nodes[snap]) return -1;
	lg_vt_entry e = t.vt[snap][v];
	for (int step = 0; step < LG_MAX_LEVELS; step++) {
		if (e.adj_list_start == LG_NIL_EDGE || e.level_length == 0) return -1;
		const uint32_t lv = LG_EDGE_LEVEL(e.adj_list_start);
		if ((int)lv < t.min_level) return -1;
		const uint64_t idx = LG_EDGE_INDEX(e.adj_list_start);
		const uint32_t* base = t.ids[lv] + idx;
		uint32_t lo = 0, hi = e.level_length;
		while (lo < hi) {
			const uint32_t mid = (lo + hi) >> 1;
			if (base[mid] < x) lo = mid + 1; else hi = mid;
		}
		if (lo < e.level_length && base[lo] == x) {
			const uint64_t k = idx + lo;
			if (!((t.del[lv][k >> 5] >> (k & 31)) & 1u)) return (int64_t)LG_EDGE_CREATE(lv, k);
		}
		if ((int)lv <= t.min_level || v >= t.max_nodes[lv - 1]) return -1;
		e = t.vt[lv - 1][v];
	}
	return -1;
}

// Deleted edges -> deletion marks of the new level `lnew`.
__global__ void bl_locate(const unsigned long long* dk, uint64_t n, BuildTab t, int snap,
		int lnew, uint2* marks, unsigned* err) {
	const uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (j >= n) return;
	const unsigned long long k = dk[j];
	const int64_t e = find_live(t, snap, (uint32_t)(k >> 32), (uint32_t)k);
	if (e < 0) { atomicOr(err, kErrNotLive); marks[j] = make_uint2(0, 0); return; }
	marks[j] = make_uint2((uint32_t)LG_EDGE_INDEX(e),
			(LG_EDGE_LEVEL(e) << LG_BITS_LEVEL) | (uint32_t)lnew);
}

__global__ void bl_not_live(const unsigned long long* k, uint64_t n, BuildTab t, int snap,
		unsigned* err) {
	const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	if (find_live(t, snap, (uint32_t)(k[i] >> 32), (uint32_t)k[i]) >= 0)
		atomicOr(err, kErrLive);
}

struct NodeOut {
	lg_vt_entry e;
	uint32_t usage;
	bool write;
};

// The element init_node (ll_mlcsr_sp.h:1375-1550) gives vertex v of level l
// with nn new edges and nd deletions; usage = slots it takes (the fragment
// and, above level 0, a two-slot continuation record); write = false keeps
// the previous level's element.  adj_list_start is 1 (placeholder) when the
// fragment starts in this level.
__device__ __forceinline__ NodeOut bl_node(uint64_t v, int l, uint32_t nn, uint32_t nd,
		const lg_vt_entry* prev, uint64_t prev_n) {
	NodeOut o;
	const bool exists_prev = l > 0 && v < prev_n;
	if (!(l == 0 || nn > 0 || nd > 0)) {
		o.e = lg_vt_entry{LG_NIL_EDGE, 0, 0};
		o.usage = 0;
		o.write = !exists_prev;
		return o;
	}
	lg_vt_entry e;
	if (l == 0 || nn > 0) {
		e.adj_list_start = nn == 0 ? LG_NIL_EDGE : 0;
		e.level_length = nn;
		e.degree = 0;
	} else if (!exists_prev) {
		e = lg_vt_entry{LG_NIL_EDGE, 0, 0};
	} else {
		e = prev[v];
	}
	uint32_t deg = nn - nd;
	if (exists_prev && prev[v].adj_list_start != LG_NIL_EDGE) deg += prev[v].degree;
	e.degree = deg;
	if (deg == 0) { e.adj_list_start = LG_NIL_EDGE; e.level_length = 0; }
	const bool cont = l > 0 && e.adj_list_start != LG_NIL_EDGE;
	o.usage = nn + (cont ? 2u : 0u);
	o.write = true;
	if (nn > 0 && e.adj_list_start != LG_NIL_EDGE) e.adj_list_start = 1;
	o.e = e;
	return o;
}

__global__ void bl_usage(uint64_t V, int l, const uint32_t* cnt, const uint32_t* dcnt,
		const lg_vt_entry* prev, uint64_t prev_n, uint32_t* usage) {
	const uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (v >= V) return;
	usage[v] = bl_node(v, l, cnt[v], dcnt ? dcnt[v] : 0u, prev, prev_n).usage;
}

__global__ void bl_place(uint64_t V, int l, const uint32_t* cnt, const uint32_t* dcnt,
		const lg_vt_entry* prev, uint64_t prev_n, const uint32_t* pos, lg_vt_entry* vt) {
	const uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (v > V) return;
	if (v == V) {   // sentinel (finish_level_vertices)
		vt[V] = lg_vt_entry{(int64_t)LG_EDGE_CREATE(l, pos[V]), 0, 0};
		return;
	}
	const uint32_t nn = cnt[v];
	NodeOut o = bl_node(v, l, nn, dcnt ? dcnt[v] : 0u, prev, prev_n);
	if (!o.write) { vt[v] = prev[v]; return; }
	if (nn > 0 && o.e.adj_list_start != LG_NIL_EDGE)
		o.e.adj_list_start = (int64_t)LG_EDGE_CREATE(l, pos[v]);
	vt[v] = o.e;
}

// New edge i (sorted keys) -> slot pos[v] + (i - off[v]).
__global__ void bl_fill(const unsigned long long* k, uint64_t n, const uint32_t* off,
		const uint32_t* pos, const uint32_t* perm, const uint32_t* w_in, uint32_t* ids,
		uint32_t* w) {
	const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	const uint32_t v = (uint32_t)(k[i] >> 32);
	const uint32_t p = pos[v] + ((uint32_t)i - off[v]);
	ids[p] = (uint32_t)k[i];
	if (w) w[p] = w_in[perm[i]];
}

// Device copy of n u32 values from host or device memory.
static lg_status to_device(lg_store* s, const uint32_t* p, uint64_t n, DevBuf& buf,
		const uint32_t** out) {
	if (n == 0) { *out = nullptr; return LG_OK; }
	if (is_device_pointer(p)) { *out = p; return LG_OK; }
	LG_TRY(buf.reserve(n * sizeof(uint32_t)));
	LG_CUDA(cudaMemcpyAsync(buf.p, p, n * sizeof(uint32_t), cudaMemcpyHostToDevice, s->stream),
			"edge delta upload");
	s->h2d_bytes += n * sizeof(uint32_t);
	*out = buf.as<uint32_t>();
	return LG_OK;
}

// Device tables of the levels of csr, with deletion bitsets of snapshot
// L = levels - 1 in `bits`.
static lg_status build_tab(lg_store* s, const DevCsr& csr, DevBuf& bits, BuildTab* t) {
	std::memset(t, 0, sizeof(*t));
	const int L = (int)csr.levels.size() - 1;
	const int m = s->min_level;
	t->min_level = m;
	if (L < 0) return LG_OK;
	std::vector<uint64_t> word_off(L + 2, 0);
	for (int l = 0; l <= L; l++)
		word_off[l + 1] = word_off[l] + (l < m ? 0 : (csr.levels[l]->n_slots + 31) / 32 + 1);
	LG_TRY(bits.reserve(std::max<uint64_t>(word_off[L + 1], 1) * sizeof(uint32_t)));
	LG_CUDA(cudaMemsetAsync(bits.p, 0, word_off[L + 1] * sizeof(uint32_t), s->stream),
			"clear deletion bits");
	for (int l = m; l <= L; l++) {
		t->vt[l] = csr.levels[l]->vt.as<lg_vt_entry>();
		t->ids[l] = csr.levels[l]->ids.as<uint32_t>();
		t->del[l] = bits.as<uint32_t>() + word_off[l];
		t->max_nodes[l] = csr.levels[l]->max_nodes;
	}
	if (csr.n_dels_dev > 0) {
		bl_mark<<<grid_for(csr.n_dels_dev, 256), 256, 0, s->stream>>>(
				csr.dels.as<uint2>(), csr.n_dels_dev, L, *t);
		LG_CUDA(cudaGetLastError(), "bl_mark");
		s->launches++;
	}
	return LG_OK;
}

// One direction's level from sorted keys (v << 32 | neighbour), the sorted
// deletion keys of the same direction, and optional weights (w_in indexed
// through perm).  The level is returned uncommitted.
static lg_status build_dir(lg_store* s, const DevCsr& csr, int l, uint64_t V,
		const unsigned long long* keys, uint64_t n, const unsigned long long* dkeys,
		uint64_t nd, const uint32_t* perm, const uint32_t* w_in, DevBuf* sc, DevLevel** out) {
	cudaStream_t st = s->stream;
	const unsigned B = 256;
	const DevLevel* prev = l > 0 ? csr.levels[l - 1] : nullptr;
	const uint64_t prev_n = prev ? prev->max_nodes : 0;
	// per-vertex counts, placement scan
	LG_TRY(sc[0].reserve(2 * V * sizeof(uint32_t)));
	uint32_t* cnt = sc[0].as<uint32_t>();
	uint32_t* dcnt = cnt + V;
	LG_CUDA(cudaMemsetAsync(cnt, 0, 2 * V * sizeof(uint32_t), st), "clear counts");
	if (n > 0) bl_count<<<grid_for(n, B), B, 0, st>>>(keys, n, cnt);
	if (nd > 0) bl_count<<<grid_for(nd, B), B, 0, st>>>(dkeys, nd, dcnt);
	LG_CUDA(cudaGetLastError(), "bl_count");
	LG_TRY(sc[1].reserve(2 * (V + 1) * sizeof(uint32_t)));
	uint32_t* off = sc[1].as<uint32_t>();
	uint32_t* usage = off + V + 1;
	LG_TRY(exclusive_scan_u32(cnt, off, V, sc[2], st, nullptr));
	const lg_vt_entry* pvt = prev ? prev->vt.as<lg_vt_entry>() : nullptr;
	bl_usage<<<grid_for(V, B), B, 0, st>>>(V, l, cnt, l > 0 ? dcnt : nullptr, pvt, prev_n, usage);
	LG_CUDA(cudaGetLastError(), "bl_usage");
	LG_TRY(sc[3].reserve((V + 1) * sizeof(uint32_t)));
	uint32_t* pos = sc[3].as<uint32_t>();
	uint64_t S = 0;
	LG_TRY(exclusive_scan_u32(usage, pos, V, sc[2], st, &S));
	if (S >= 0xffffffffull)
		return set_error(LG_ENOTSUP, "more than 2^32-1 slots in one level");

	DevLevel* d = take_level(s, &csr == &s->out ? 0 : 1);
	if (!d) return set_error(LG_ENOMEM, "host allocation");
	d->max_nodes = V;
	d->n_slots = S;
	d->n_fragment_slots = n;
	if (!w_in) d->w.release();
	lg_status rs = d->vt.reserve((V + 1) * sizeof(lg_vt_entry));
	if (!rs) rs = d->ids.reserve(std::max<uint64_t>(S, 1) * sizeof(uint32_t));
	if (!rs && w_in) rs = d->w.reserve(std::max<uint64_t>(S, 1) * sizeof(uint32_t));
	if (rs) { delete d; return rs; }
	cudaError_t ce = cudaMemsetAsync(d->ids.p, 0xff, std::max<uint64_t>(S, 1) * sizeof(uint32_t), st);
	if (ce == cudaSuccess && w_in)
		ce = cudaMemsetAsync(d->w.p, 0, std::max<uint64_t>(S, 1) * sizeof(uint32_t), st);
	if (ce != cudaSuccess) { delete d; return cuda_status(ce, "clear level"); }
	bl_place<<<grid_for(V + 1, B), B, 0, st>>>(V, l, cnt, l > 0 ? dcnt : nullptr, pvt, prev_n,
			pos, d->vt.as<lg_vt_entry>());
	if (n > 0)
		bl_fill<<<grid_for(n, B), B, 0, st>>>(keys, n, off, pos, perm, w_in,
				d->ids.as<uint32_t>(), w_in ? d->w.as<uint32_t>() : nullptr);
	ce = cudaGetLastError();
	if (ce != cudaSuccess) { delete d; return cuda_status(ce, "bl_place"); }
	s->launches += 2 + (n > 0) + (nd > 0) + 3 + 1 + 3 + (n > 0);
	*out = d;
	return LG_OK;
}

// Sorted (a << 32 | b) keys of n pairs (payload = input index when `perm`)
// in `keys`; err gets kErrRange / dup_bit.
static lg_status sorted_keys(lg_store* s, const uint32_t* a, const uint32_t* b, uint64_t n,
		uint64_t V, bool perm, unsigned dup_bit, unsigned* err, DevBuf& keys_buf,
		DevBuf& perm_buf, DevBuf* tmp, unsigned long long** keys, uint32_t** perm_out) {
	cudaStream_t st = s->stream;
	const unsigned B = 256;
	*keys = nullptr;
	if (perm_out) *perm_out = nullptr;
	if (n == 0) return LG_OK;
	LG_TRY(keys_buf.reserve(n * sizeof(unsigned long long)));
	if (perm) LG_TRY(perm_buf.reserve(n * sizeof(uint32_t)));
	bl_keys<<<grid_for(n, B), B, 0, st>>>(a, b, n, V, keys_buf.as<unsigned long long>(),
			perm ? perm_buf.as<uint32_t>() : nullptr, err);
	LG_CUDA(cudaGetLastError(), "bl_keys");
	s->launches++;
	unsigned long long* sk = nullptr;
	uint32_t* sp = nullptr;
	LG_TRY(radix_sort_u64(s, keys_buf.as<unsigned long long>(),
			perm ? perm_buf.as<uint32_t>() : nullptr, n, tmp[0], tmp[1], tmp[2], tmp[3], &sk, &sp));
	// keep the result in keys_buf / perm_buf (the temporaries are reused)
	if (sk != keys_buf.as<unsigned long long>())
		LG_CUDA(cudaMemcpyAsync(keys_buf.p, sk, n * sizeof(unsigned long long),
				cudaMemcpyDeviceToDevice, st), "sorted keys");
	if (perm && sp != perm_buf.as<uint32_t>())
		LG_CUDA(cudaMemcpyAsync(perm_buf.p, sp, n * sizeof(uint32_t),
				cudaMemcpyDeviceToDevice, st), "sorted payload");
	bl_dups<<<grid_for(n, B), B, 0, st>>>(keys_buf.as<unsigned long long>(), n, err, dup_bit);
	LG_CUDA(cudaGetLastError(), "bl_dups");
	s->launches++;
	*keys = keys_buf.as<unsigned long long>();
	if (perm_out) *perm_out = perm ? perm_buf.as<uint32_t>() : nullptr;
	return LG_OK;
}

} // namespace lg

using namespace lg;

extern "C" lg_status lg_store_build_level(lg_store* s, uint64_t max_nodes,
		const uint32_t* src, const uint32_t* dst, const uint32_t* weights, uint64_t n_new,
		const uint32_t* del_src, const uint32_t* del_dst, uint64_t n_del) {
	clear_error();
	if (!s) return set_error(LG_EINVAL, "null store");
	const int l = (int)s->out.levels.size();
	if (l >= LG_MAX_LEVELS) return set_error(LG_ENOTSUP, "more than %d levels", LG_MAX_LEVELS);
	if (max_nodes == 0 || max_nodes >= 0xffffffffull)
		return set_error(LG_EINVAL, "max_nodes must be in [1, 2^32-1)");
	if (l > 0 && max_nodes < s->out.levels[l - 1]->max_nodes)
		return set_error(LG_EINVAL, "max_nodes cannot shrink");
	if (l == 0 && n_del > 0) return set_error(LG_EINVAL, "level 0 cannot delete edges");
	if (n_new > 0 && (!src || !dst)) return set_error(LG_EINVAL, "null edge array");
	if (n_del > 0 && (!del_src || !del_dst)) return set_error(LG_EINVAL, "null deletion array");
	if (n_new >= 0xffffffffull || n_del >= 0xffffffffull)
		return set_error(LG_ENOTSUP, "more than 2^32-1 edges in one delta");
	LG_CUDA(cudaSetDevice(s->device), "cudaSetDevice");
	cudaStream_t st = s->stream;
	const uint64_t V = max_nodes;
	DevBuf* sc = s->scratch;
	const unsigned B = 256;

	// inputs on the device
	const uint32_t *ds = nullptr, *dd = nullptr, *dw = nullptr, *xs = nullptr, *xd = nullptr;
	DevBuf* up = s->build_tmp;          // uploads of host inputs
	LG_TRY(to_device(s, src, n_new, up[0], &ds));
	LG_TRY(to_device(s, dst, n_new, up[1], &dd));
	if (weights) LG_TRY(to_device(s, weights, n_new, up[2], &dw));
	LG_TRY(to_device(s, del_src, n_del, up[3], &xs));
	LG_TRY(to_device(s, del_dst, n_del, up[4], &xd));
	LG_TRY(sc[11].reserve(sizeof(unsigned)));
	unsigned* err = sc[11].as<unsigned>();
	LG_CUDA(cudaMemsetAsync(err, 0, sizeof(unsigned), st), "clear flag");

	// out direction: sorted new edges (weights follow) and deletions
	DevBuf& ok_keys = s->build_tmp[5];
	DevBuf& ok_perm = s->build_tmp[6];
	DevBuf& od_keys = s->build_tmp[7];
	DevBuf& bits = s->build_tmp[8];
	unsigned long long *ok = nullptr, *od = nullptr;
	uint32_t* operm = nullptr;
	LG_TRY(sorted_keys(s, ds, dd, n_new, V, weights != nullptr, kErrDupNew, err, ok_keys,
			ok_perm, sc + 4, &ok, &operm));
	LG_TRY(sorted_keys(s, xs, xd, n_del, V, false, kErrDupDel, err, od_keys, ok_perm,
			sc + 4, &od, nullptr));
	DevBuf& marks = s->build_tmp[9];
	LG_TRY(marks.reserve(std::max<uint64_t>(2 * n_del, 1) * sizeof(uint2)));
	if (l > 0) {
		BuildTab t;
		LG_TRY(build_tab(s, s->out, bits, &t));
		if (n_del > 0)
			bl_locate<<<grid_for(n_del, B), B, 0, st>>>(od, n_del, t, l - 1, l,
					marks.as<uint2>(), err);
		if (n_new > 0)
			bl_not_live<<<grid_for(n_new, B), B, 0, st>>>(ok, n_new, t, l - 1, err);
		LG_CUDA(cudaGetLastError(), "bl_locate");
		s->launches += (n_del > 0) + (n_new > 0);
	}
	DevLevel* lo = nullptr;
	DevLevel* li = nullptr;
	LG_TRY(build_dir(s, s->out, l, V, ok, n_new, od, n_del, operm, dw, sc, &lo));

	// in direction: the same edges keyed by target (sources stay sorted
	// within a target, as make_reverse_edges leaves them)
	lg_status rs = LG_OK;
	if (s->reverse) {
		DevBuf& ik_keys = s->build_tmp[10];
		DevBuf& id_keys = s->build_tmp[11];
		unsigned long long *ik = nullptr, *idk = nullptr;
		if (n_new > 0) {
			rs = ik_keys.reserve(n_new * sizeof(unsigned long long));
			if (!rs) {
				bl_swap<<<grid_for(n_new, B), B, 0, st>>>(ok, n_new, ik_keys.as<unsigned long long>());
				unsigned long long* sk = nullptr;
				uint32_t* sp = nullptr;
				rs = radix_sort_u64(s, ik_keys.as<unsigned long long>(), nullptr, n_new,
						sc[4], sc[5], sc[6], sc[7], &sk, &sp);
				ik = sk;
			}
		}
		if (!rs && n_del > 0) {
			rs = id_keys.reserve(n_del * sizeof(unsigned long long));
			if (!rs) {
				bl_swap<<<grid_for(n_del, B), B, 0, st>>>(od, n_del, id_keys.as<unsigned long long>());
				unsigned long long* sk = nullptr;
				uint32_t* sp = nullptr;
				rs = radix_sort_u64(s, id_keys.as<unsigned long long>(), nullptr, n_del,
						sc[8], sc[9], sc[10], sc[2], &sk, &sp);
				idk = sk;
			}
		}
		s->launches += (n_new > 0) + (n_del > 0);
		if (!rs && l > 0 && n_del > 0) {
			BuildTab t;
			rs = build_tab(s, s->in, bits, &t);
			if (!rs) {
				bl_locate<<<grid_for(n_del, B), B, 0, st>>>(idk, n_del, t, l - 1, l,
						marks.as<uint2>() + n_del, err);
				s->launches++;
			}
		}
		if (!rs) rs = build_dir(s, s->in, l, V, ik, n_new, idk, n_del, nullptr, nullptr, sc, &li);
		if (!rs) {
			// ik / idk may live in the sort temporaries: finish before they go
			const cudaError_t ce = cudaStreamSynchronize(st);
			if (ce != cudaSuccess) rs = cuda_status(ce, "build level");
		}
	}
	unsigned herr = 0;
	if (!rs) {
		cudaError_t ce = cudaMemcpyAsync(&herr, err, sizeof(herr), cudaMemcpyDeviceToHost, st);
		if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
		if (ce != cudaSuccess) rs = cuda_status(ce, "build level");
		s->d2h_bytes += sizeof(herr);
	}
	if (!rs && herr) {
		if (herr & kErrRange) rs = set_error(LG_EINVAL, "vertex id out of range");
		else if (herr & kErrDupNew) rs = set_error(LG_EINVAL, "duplicate new edge");
		else if (herr & kErrDupDel) rs = set_error(LG_EINVAL, "edge deleted twice");
		else if (herr & kErrNotLive) rs = set_error(LG_EINVAL, "deleted edge is not live");
		else rs = set_error(LG_EINVAL, "new edge is already live");
	}
	if (rs) {
		cudaStreamSynchronize(st);
		delete lo;
		delete li;
		return rs;
	}
	// commit
	s->out.levels.push_back(lo);
	// the deletion marks go from the build buffer to the lists, on the device
	LG_TRY(append_dels(s, s->out, marks.as<uint2>(), n_del, cudaMemcpyDeviceToDevice));
	if (s->reverse) {
		s->in.levels.push_back(li);
		LG_TRY(append_dels(s, s->in, marks.as<uint2>() + n_del, n_del, cudaMemcpyDeviceToDevice));
	}
	LG_CUDA(cudaStreamSynchronize(st), "build level");
	return LG_OK;
}

extern "C" lg_status lg_store_read_level(lg_store* s, int level, int dir, lg_vt_entry* vt,
		uint32_t* ids, uint32_t* weights, uint64_t* n_slots) {
	clear_error();
	if (!s) return set_error(LG_EINVAL, "null store");
	if (dir != 0 && dir != 1) return set_error(LG_EINVAL, "dir must be 0 or 1");
	const DevCsr& csr = dir == 0 ? s->out : s->in;
	if (dir == 1 && !s->reverse) return set_error(LG_ESTATE, "the store has no in-CSR");
	if (level < 0 || level >= (int)csr.levels.size())
		return set_error(LG_EINVAL, "level %d out of range", level);
	const DevLevel* d = csr.levels[level];
	if (level < s->min_level) return set_error(LG_ESTATE, "level %d is aged out", level);
	if (weights && !d->w.p) return set_error(LG_ESTATE, "the level has no edge weights");
	LG_CUDA(cudaSetDevice(s->device), "cudaSetDevice");
	if (n_slots) *n_slots = d->n_slots;
	if (vt) LG_TRY(copy_out(s, vt, d->vt.p, (d->max_nodes + 1) * sizeof(lg_vt_entry)));
	if (ids) LG_TRY(copy_out(s, ids, d->ids.p, d->n_slots * sizeof(uint32_t)));
	if (weights) LG_TRY(copy_out(s, weights, d->w.p, d->n_slots * sizeof(uint32_t)));
	LG_CUDA(cudaStreamSynchronize(s->stream), "read level");
	return LG_OK;
}
