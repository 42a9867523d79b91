// lg_host.cpp - host-side level construction and seeded graph generators.
//
// Level construction follows the reference's read-only level builder:
//   init_level_from_degrees  llama/include/llama/ll_mlcsr_sp.h:1562-1607
//   init_node                llama/include/llama/ll_mlcsr_sp.h:1375-1550
//   write_value(s)           llama/include/llama/ll_mlcsr_sp.h:1618-1715
//   finish_level_vertices    llama/include/llama/ll_mlcsr_sp.h:786-808
//   update_max_visible_level_lower_only  llama/include/llama/ll_mlcsr_sp.h:849-863
// and produces byte-identical vertex tables and edge-table slots (checked
// against the reference itself by the test suite).  The reference walks the
// vertices one by one; here the per-vertex slot usage is computed first and
// a parallel prefix sum places every fragment, which yields the same layout
// because the reference also places fragments in vertex order.
//
// Sizing note: the reference sizes a level's continuation space by counting
// only vertices with new edges (ll_mlcsr_sp.h:1575-1578) while init_node also
// writes a continuation for deletion-only vertices (ll_mlcsr_sp.h:1474-1497).
// Here every slot is counted, so the layout is the one init_node writes.

#include "lg_internal.h"
#include "../../include/lg_host.h"

#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

namespace lg {

// ---------------------------------------------------------------------------
// Parallel helpers
// ---------------------------------------------------------------------------

// Exclusive prefix sum of in[0..n) into out[0..n]; returns the total.
static uint64_t parallel_exclusive_scan(const uint32_t* in, uint64_t* out,
		uint64_t n) {
	int nt = omp_get_max_threads();
	std::vector<uint64_t> part(nt + 1, 0);
#pragma omp parallel num_threads(nt)
	{
		int t = omp_get_thread_num();
		uint64_t lo = n * t / nt, hi = n * (t + 1) / nt, s = 0;
		for (uint64_t i = lo; i < hi; i++) s += in[i];
		part[t + 1] = s;
#pragma omp barrier
#pragma omp single
		for (int k = 0; k < nt; k++) part[k + 1] += part[k];
		uint64_t acc = part[t];
		for (uint64_t i = lo; i < hi; i++) { out[i] = acc; acc += in[i]; }
	}
	out[n] = part[nt];
	return part[nt];
}

// LSD radix sort of 64-bit keys (with an optional 32-bit payload), 8-bit
// digits, skipping digits that are constant over the input.
static void radix_sort_u64(std::vector<uint64_t>& keys,
		std::vector<uint32_t>* payload) {
	uint64_t n = keys.size();
	if (n < 2) return;
	int nt = omp_get_max_threads();
	uint64_t all_or = 0, all_and = ~0ull;
#pragma omp parallel for reduction(|:all_or) reduction(&:all_and) num_threads(nt)
	for (uint64_t i = 0; i < n; i++) { all_or |= keys[i]; all_and &= keys[i]; }
	uint64_t varying = all_or ^ all_and;
	std::vector<uint64_t> tmp(n);
	std::vector<uint32_t> ptmp;
	if (payload) ptmp.resize(n);
	std::vector<uint64_t> hist((size_t)nt * 256);
	for (int shift = 0; shift < 64; shift += 8) {
		if (((varying >> shift) & 0xff) == 0) continue;
		std::fill(hist.begin(), hist.end(), 0);
#pragma omp parallel num_threads(nt)
		{
			int t = omp_get_thread_num();
			uint64_t lo = n * t / nt, hi = n * (t + 1) / nt;
			uint64_t* h = &hist[(size_t)t * 256];
			for (uint64_t i = lo; i < hi; i++) h[(keys[i] >> shift) & 0xff]++;
#pragma omp barrier
#pragma omp single
			{
				uint64_t s = 0;
				for (int d = 0; d < 256; d++)
					for (int k = 0; k < nt; k++) {
						uint64_t c = hist[(size_t)k * 256 + d];
						hist[(size_t)k * 256 + d] = s;
						s += c;
					}
			}
			for (uint64_t i = lo; i < hi; i++) {
				uint64_t pos = h[(keys[i] >> shift) & 0xff]++;
				tmp[pos] = keys[i];
				if (payload) ptmp[pos] = (*payload)[i];
			}
		}
		keys.swap(tmp);
		if (payload) payload->swap(ptmp);
	}
}

static bool is_sorted_parallel(const std::vector<uint64_t>& k) {
	uint64_t n = k.size();
	int bad = 0;
#pragma omp parallel for reduction(|:bad)
	for (uint64_t i = 1; i < n; i++) bad |= (k[i - 1] > k[i]);
	return !bad;
}

// ---------------------------------------------------------------------------
// Seeded hashing (splitmix64 finaliser), used for every random choice so that
// results do not depend on the thread count.
// ---------------------------------------------------------------------------

static inline uint64_t mix64(uint64_t z) {
	z += 0x9e3779b97f4a7c15ull;
	z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
	z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
	return z ^ (z >> 31);
}
static inline double unit_double(uint64_t h) {   // [0, 1), 53 bits
	return (double)(h >> 11) * (1.0 / 9007199254740992.0);
}
static inline uint64_t canon_key(uint32_t s, uint32_t t, int symmetric) {
	if (symmetric && t < s) std::swap(s, t);
	return ((uint64_t)s << 32) | t;
}

// Bijective scramble of [0, 2^scale) for Kronecker vertex ids.
static inline uint32_t scramble_id(uint64_t x, int scale, uint64_t seed) {
	uint64_t mask = (scale >= 64) ? ~0ull : ((1ull << scale) - 1);
	uint64_t k1 = mix64(seed ^ 0x1234567ull) | 1ull;
	uint64_t k2 = mix64(seed ^ 0x89abcdefull);
	uint64_t k3 = mix64(seed ^ 0x13579bdfull) | 1ull;
	int half = scale / 2 > 0 ? scale / 2 : 1;
	x = (x * k1 + k2) & mask;
	x ^= x >> half;
	x = (x * k3) & mask;
	x ^= x >> half;
	x = (x * k1 + (k2 >> 7)) & mask;
	return (uint32_t)x;
}

static inline void rmat_draw(uint64_t seed, uint64_t i, int scale, double a,
		double ab, double abc, uint32_t* s, uint32_t* t) {
	uint64_t state = mix64(seed * 0x2545f4914f6cdd1dull + i);
	uint32_t u = 0, v = 0;
	for (int k = 0; k < scale; k++) {
		state = mix64(state);
		double r = unit_double(state);
		uint32_t row, col;
		if (r < a) { row = 0; col = 0; }
		else if (r < ab) { row = 0; col = 1; }
		else if (r < abc) { row = 1; col = 0; }
		else { row = 1; col = 1; }
		u = (u << 1) | row;
		v = (v << 1) | col;
	}
	*s = u; *t = v;
}

// ---------------------------------------------------------------------------
// Host multiversion graph
// ---------------------------------------------------------------------------

struct HCsr {
	std::vector<std::vector<lg_vt_entry>> vt;       // per level, max_nodes + 1
	std::vector<std::vector<uint64_t>> slots;       // per level
	std::vector<std::vector<uint32_t>> weights;     // per level (may be empty)
	std::vector<std::vector<lg_deletion>> dels;     // marks made by the level
};

struct LevelInput {
	std::vector<uint32_t> src, dst, dsrc, ddst, w;
};

} // namespace lg

struct lg_hgraph {
	uint64_t V;
	int rev;
	lg::HCsr out, in;
	std::vector<lg::LevelInput> inputs;
};

namespace lg {

// Find the slot holding (v -> t) live in snapshot `snap` by walking v's
// fragment chain exactly as iter_begin/iter_descend do
// (llama/include/llama/ll_mlcsr_sp.h:1994-2134); fragments are sorted by
// payload, so each is binary searched.  Returns the edge id or -1.
static int64_t find_live_slot(const HCsr& c, int snap, uint64_t v, uint32_t t) {
	if (v + 1 >= c.vt[snap].size()) return -1;
	lg_vt_entry e = c.vt[snap][v];
	while (true) {
		if (e.adj_list_start == LG_NIL_EDGE || e.level_length == 0) return -1;
		uint32_t lv = LG_EDGE_LEVEL(e.adj_list_start);
		uint64_t idx = LG_EDGE_INDEX(e.adj_list_start);
		const uint64_t* base = c.slots[lv].data() + idx;
		uint64_t lo = 0, hi = e.level_length;
		while (lo < hi) {
			uint64_t mid = (lo + hi) / 2;
			if (LG_SLOT_PAYLOAD(base[mid]) < t) lo = mid + 1; else hi = mid;
		}
		if (lo < e.level_length && LG_SLOT_PAYLOAD(base[lo]) == t
				&& LG_SLOT_MAX_LEVEL(base[lo]) > (uint32_t)snap)
			return LG_EDGE_CREATE(lv, idx + lo);
		if (lv == 0 || v + 1 >= c.vt[lv - 1].size()) return -1;
		e = c.vt[lv - 1][v];
	}
}

// Build level `l` of one CSR.  nbr: neighbours of the new edges grouped by
// vertex (off[v]..off[v+1]) and sorted; del_cnt: deletions per vertex at this
// level; w: per-new-edge weights aligned with nbr (or NULL).
static void build_csr_level(HCsr& c, int l, uint64_t V, const uint32_t* nbr,
		const uint64_t* off, const uint32_t* del_cnt, const uint32_t* w,
		bool want_weights) {
	c.vt.emplace_back();   // (may reallocate c.vt: take references after it)
	std::vector<lg_vt_entry>* prev = l > 0 ? &c.vt[l - 1] : nullptr;
	uint64_t prev_n = prev ? prev->size() - 1 : 0;  // max_nodes of level l-1
	std::vector<lg_vt_entry>& vt = c.vt.back();
	if (prev) {
		vt.resize(V + 1);
		uint64_t m = std::min<uint64_t>(prev_n, V);
#pragma omp parallel for schedule(static)
		for (uint64_t v = 0; v < m; v++) vt[v] = (*prev)[v];
		// Vertices that did not exist in the previous level start as zeroed
		// elements; init_node turns the untouched ones into NIL below.
		for (uint64_t v = m; v <= V; v++) { vt[v] = lg_vt_entry{0, 0, 0}; }
	} else {
		vt.assign(V + 1, lg_vt_entry{LG_NIL_EDGE, 0, 0});
	}

	// Pass 1: the element each vertex gets and the slots it consumes
	// (init_node, ll_mlcsr_sp.h:1375-1550).
	std::vector<lg_vt_entry> ne(V);
	std::vector<uint32_t> usage(V);
	std::vector<uint8_t> write(V);
#pragma omp parallel for schedule(static)
	for (uint64_t v = 0; v < V; v++) {
		uint64_t nn = off[v + 1] - off[v];
		uint64_t nd = (l == 0 || !del_cnt) ? 0 : del_cnt[v];
		bool exists_prev = l > 0 && v < prev_n;
		if (!(l == 0 || nn > 0 || nd > 0)) {
			usage[v] = 0;
			write[v] = !exists_prev;   // NIL for vertices new to this level
			ne[v] = lg_vt_entry{LG_NIL_EDGE, 0, 0};
			continue;
		}
		lg_vt_entry e;
		if (l == 0 || nn > 0) {
			e.adj_list_start = nn == 0 ? LG_NIL_EDGE : 0;  // placed in pass 2
			e.level_length = (uint32_t)nn;
			e.degree = 0;
		} else if (!exists_prev) {
			e = lg_vt_entry{LG_NIL_EDGE, 0, 0};
		} else {
			e = (*prev)[v];
		}
		uint32_t deg = (uint32_t)(nn - nd);
		if (exists_prev && (*prev)[v].adj_list_start != LG_NIL_EDGE)
			deg += (*prev)[v].degree;
		e.degree = deg;
		if (deg == 0) { e.adj_list_start = LG_NIL_EDGE; e.level_length = 0; }
		bool cont = l > 0 && e.adj_list_start != LG_NIL_EDGE;
		usage[v] = (uint32_t)(nn + (cont ? 2 : 0));
		write[v] = 1;
		// mark "starts in this level" with a non-NIL placeholder
		if (nn > 0 && e.adj_list_start != LG_NIL_EDGE) e.adj_list_start = 1;
		ne[v] = e;
	}

	// Pass 2: place fragments in vertex order.
	std::vector<uint64_t> pos(V + 1);
	uint64_t total = parallel_exclusive_scan(usage.data(), pos.data(), V);
	c.slots.emplace_back(total, 0ull);
	std::vector<uint64_t>& sl = c.slots.back();
	c.weights.emplace_back();
	std::vector<uint32_t>* wl = nullptr;
	if (want_weights) { c.weights.back().assign(total, 0u); wl = &c.weights.back(); }

#pragma omp parallel for schedule(dynamic, 4096)
	for (uint64_t v = 0; v < V; v++) {
		if (!write[v]) continue;
		lg_vt_entry e = ne[v];
		uint64_t nn = off[v + 1] - off[v];
		uint64_t p = pos[v];
		if (nn > 0 && e.adj_list_start != LG_NIL_EDGE)
			e.adj_list_start = LG_EDGE_CREATE(l, p);
		for (uint64_t k = 0; k < nn; k++) {
			sl[p + k] = (uint64_t)nbr[off[v] + k]
				| ((uint64_t)LG_FRESH_MAX_LEVEL << LG_BITS_INDEX);
			if (wl) (*wl)[p + k] = w ? w[off[v] + k] : 0u;
		}
		if (l > 0 && e.adj_list_start != LG_NIL_EDGE) {
			// continuation record: the previous level's element of v
			lg_vt_entry b = (v < prev_n) ? (*prev)[v]
				: lg_vt_entry{LG_NIL_EDGE, 0, 0};
			std::memcpy(&sl[p + nn], &b, sizeof(b));
		}
		vt[v] = e;
	}
	// sentinel (finish_level_vertices)
	vt[V] = lg_vt_entry{LG_EDGE_CREATE(l, total), 0, 0};
}

static lg_status add_level_impl(lg_hgraph* g, const uint32_t* src,
		const uint32_t* dst, uint64_t n_new, const uint32_t* dsrc,
		const uint32_t* ddst, uint64_t n_del, const uint32_t* weights) {
	const uint64_t V = g->V;
	const int l = (int)g->out.vt.size();
	if (l >= LG_MAX_LEVELS) return set_error(LG_ENOTSUP, "too many levels");
	if (l == 0 && n_del > 0)
		return set_error(LG_EINVAL, "level 0 cannot delete edges");
	int bad = 0;
#pragma omp parallel for reduction(|:bad)
	for (uint64_t i = 0; i < n_new; i++)
		bad |= (src[i] >= V || dst[i] >= V);
#pragma omp parallel for reduction(|:bad)
	for (uint64_t i = 0; i < n_del; i++)
		bad |= (dsrc[i] >= V || ddst[i] >= V);
	if (bad) return set_error(LG_EINVAL, "vertex id out of range");

	// Keep the inputs (sorted) for lg_hgraph_level_input.
	LevelInput in;
	{
		std::vector<uint64_t> keys(n_new);
		std::vector<uint32_t> idx;
#pragma omp parallel for
		for (uint64_t i = 0; i < n_new; i++)
			keys[i] = ((uint64_t)src[i] << 32) | dst[i];
		if (!is_sorted_parallel(keys)) {
			if (weights) {
				idx.resize(n_new);
#pragma omp parallel for
				for (uint64_t i = 0; i < n_new; i++) idx[i] = (uint32_t)i;
			}
			radix_sort_u64(keys, weights ? &idx : nullptr);
		}
		for (uint64_t i = 1; i < n_new; i++)
			if (keys[i] == keys[i - 1])
				return set_error(LG_EINVAL, "duplicate new edge");
		in.src.resize(n_new); in.dst.resize(n_new);
		if (weights) in.w.resize(n_new);
#pragma omp parallel for
		for (uint64_t i = 0; i < n_new; i++) {
			in.src[i] = (uint32_t)(keys[i] >> 32);
			in.dst[i] = (uint32_t)keys[i];
			if (weights) in.w[i] = weights[idx.empty() ? i : idx[i]];
		}
		std::vector<uint64_t> dk(n_del);
#pragma omp parallel for
		for (uint64_t i = 0; i < n_del; i++)
			dk[i] = ((uint64_t)dsrc[i] << 32) | ddst[i];
		if (!is_sorted_parallel(dk)) radix_sort_u64(dk, nullptr);
		in.dsrc.resize(n_del); in.ddst.resize(n_del);
#pragma omp parallel for
		for (uint64_t i = 0; i < n_del; i++) {
			in.dsrc[i] = (uint32_t)(dk[i] >> 32);
			in.ddst[i] = (uint32_t)dk[i];
		}
	}

	// Locate the deleted edges in the latest snapshot (out and in CSR) and
	// check that new edges are not live already.
	std::vector<int64_t> del_out(n_del), del_in(g->rev ? n_del : 0);
	if (l > 0) {
#pragma omp parallel for reduction(|:bad)
		for (uint64_t i = 0; i < n_del; i++) {
			del_out[i] = find_live_slot(g->out, l - 1, in.dsrc[i], in.ddst[i]);
			bad |= del_out[i] < 0;
			if (g->rev) {
				del_in[i] = find_live_slot(g->in, l - 1, in.ddst[i], in.dsrc[i]);
				bad |= del_in[i] < 0;
			}
		}
		if (bad) return set_error(LG_EINVAL, "deleted edge is not live");
		for (uint64_t i = 1; i < n_del; i++)
			if (in.dsrc[i] == in.dsrc[i - 1] && in.ddst[i] == in.ddst[i - 1])
				return set_error(LG_EINVAL, "edge deleted twice");
#pragma omp parallel for reduction(|:bad)
		for (uint64_t i = 0; i < n_new; i++)
			bad |= find_live_slot(g->out, l - 1, in.src[i], in.dst[i]) >= 0;
		if (bad) return set_error(LG_EINVAL, "new edge is already live");
	}

	// Out-CSR level.
	{
		std::vector<uint64_t> off(V + 1);
		std::vector<uint32_t> cnt(V, 0), dcnt(V, 0);
		for (uint64_t i = 0; i < n_new; i++) cnt[in.src[i]]++;
		for (uint64_t i = 0; i < n_del; i++) dcnt[in.dsrc[i]]++;
		parallel_exclusive_scan(cnt.data(), off.data(), V);
		build_csr_level(g->out, l, V, in.dst.data(), off.data(), dcnt.data(),
				weights ? in.w.data() : nullptr, weights != nullptr);
	}
	// In-CSR level: new edges regrouped by target (stable, so sources stay
	// sorted within each target).
	if (g->rev) {
		std::vector<uint64_t> off(V + 1);
		std::vector<uint32_t> cnt(V, 0), dcnt(V, 0);
		for (uint64_t i = 0; i < n_new; i++) cnt[in.dst[i]]++;
		for (uint64_t i = 0; i < n_del; i++) dcnt[in.ddst[i]]++;
		parallel_exclusive_scan(cnt.data(), off.data(), V);
		std::vector<uint32_t> nbr(n_new);
		std::vector<uint64_t> fill(off.begin(), off.end() - 1);
		for (uint64_t i = 0; i < n_new; i++) nbr[fill[in.dst[i]]++] = in.src[i];
		build_csr_level(g->in, l, V, nbr.data(), off.data(), dcnt.data(),
				nullptr, false);
	}

	// Deletion marks in older slots (lower-only).
	g->out.dels.emplace_back(n_del);
	if (g->rev) g->in.dels.emplace_back(n_del);
#pragma omp parallel for
	for (uint64_t i = 0; i < n_del; i++) {
		int64_t e = del_out[i];
		uint64_t& s = g->out.slots[LG_EDGE_LEVEL(e)][LG_EDGE_INDEX(e)];
		if ((uint32_t)l < LG_SLOT_MAX_LEVEL(s))
			s = LG_SLOT_PAYLOAD(s) | ((uint64_t)l << LG_BITS_INDEX);
		g->out.dels.back()[i] = lg_deletion{e, (uint32_t)l, 0};
		if (g->rev) {
			int64_t f = del_in[i];
			uint64_t& r = g->in.slots[LG_EDGE_LEVEL(f)][LG_EDGE_INDEX(f)];
			if ((uint32_t)l < LG_SLOT_MAX_LEVEL(r))
				r = LG_SLOT_PAYLOAD(r) | ((uint64_t)l << LG_BITS_INDEX);
			g->in.dels.back()[i] = lg_deletion{f, (uint32_t)l, 0};
		}
	}
	g->inputs.push_back(std::move(in));
	return LG_OK;
}

} // namespace lg

using namespace lg;

extern "C" {

lg_status lg_hgraph_create(lg_hgraph** g, uint64_t max_nodes, int reverse_edges) {
	clear_error();
	if (!g) return set_error(LG_EINVAL, "null output pointer");
	if (max_nodes == 0 || max_nodes >= 0xffffffffull)
		return set_error(LG_EINVAL, "max_nodes must be in [1, 2^32-1)");
	lg_hgraph* h = new (std::nothrow) lg_hgraph();
	if (!h) return set_error(LG_ENOMEM, "out of host memory");
	h->V = max_nodes;
	h->rev = reverse_edges ? 1 : 0;
	*g = h;
	return LG_OK;
}

lg_status lg_hgraph_destroy(lg_hgraph* g) {
	delete g;
	return LG_OK;
}

lg_status lg_hgraph_add_level(lg_hgraph* g, const uint32_t* src,
		const uint32_t* dst, uint64_t n_new, const uint32_t* del_src,
		const uint32_t* del_dst, uint64_t n_del, const uint32_t* weights) {
	clear_error();
	if (!g) return set_error(LG_EINVAL, "null graph");
	if ((n_new && (!src || !dst)) || (n_del && (!del_src || !del_dst)))
		return set_error(LG_EINVAL, "null edge arrays");
	try {
		return add_level_impl(g, src, dst, n_new, del_src, del_dst, n_del,
				weights);
	} catch (const std::bad_alloc&) {
		return set_error(LG_ENOMEM, "out of host memory building a level");
	}
}

int lg_hgraph_num_levels(const lg_hgraph* g) {
	return g ? (int)g->out.vt.size() : 0;
}

uint64_t lg_hgraph_max_nodes(const lg_hgraph* g) { return g ? g->V : 0; }

lg_status lg_hgraph_level_desc(lg_hgraph* g, int level, lg_level_desc* d) {
	clear_error();
	if (!g || !d) return set_error(LG_EINVAL, "null argument");
	if (level < 0 || level >= (int)g->out.vt.size())
		return set_error(LG_EINVAL, "no such level");
	std::memset(d, 0, sizeof(*d));
	d->out.max_nodes = g->out.vt[level].size() - 1;
	d->out.vt = g->out.vt[level].data();
	d->out.n_slots = g->out.slots[level].size();
	d->out.slots = g->out.slots[level].data();
	d->out.weights = g->out.weights[level].empty() ? nullptr
		: g->out.weights[level].data();
	d->out_deletions = g->out.dels[level].data();
	d->n_out_deletions = g->out.dels[level].size();
	if (g->rev) {
		d->in.max_nodes = g->in.vt[level].size() - 1;
		d->in.vt = g->in.vt[level].data();
		d->in.n_slots = g->in.slots[level].size();
		d->in.slots = g->in.slots[level].data();
		d->in_deletions = g->in.dels[level].data();
		d->n_in_deletions = g->in.dels[level].size();
	}
	return LG_OK;
}

lg_status lg_hgraph_ingest(lg_hgraph* g, lg_store* store, int first) {
	clear_error();
	if (!g || !store) return set_error(LG_EINVAL, "null argument");
	if (first != lg_store_num_levels(store))
		return set_error(LG_ESTATE, "store does not hold exactly the levels before `first`");
	for (int l = first; l < (int)g->out.vt.size(); l++) {
		lg_level_desc d;
		lg_status st = lg_hgraph_level_desc(g, l, &d);
		if (st) return st;
		st = lg_store_ingest_level(store, &d);
		if (st) return st;
	}
	return LG_OK;
}

lg_status lg_hgraph_level_input(lg_hgraph* g, int level, const uint32_t** src,
		const uint32_t** dst, uint64_t* n_new, const uint32_t** del_src,
		const uint32_t** del_dst, uint64_t* n_del, const uint32_t** weights) {
	clear_error();
	if (!g || level < 0 || level >= (int)g->inputs.size())
		return set_error(LG_EINVAL, "no such level");
	const LevelInput& in = g->inputs[level];
	if (src) *src = in.src.data();
	if (dst) *dst = in.dst.data();
	if (n_new) *n_new = in.src.size();
	if (del_src) *del_src = in.dsrc.data();
	if (del_dst) *del_dst = in.ddst.data();
	if (n_del) *n_del = in.dsrc.size();
	if (weights) *weights = in.w.empty() ? nullptr : in.w.data();
	return LG_OK;
}

uint32_t lg_gen_weight(const lg_graph_spec* s, uint32_t src, uint32_t dst) {
	if (!s || s->weight_max == 0) return 0;
	uint64_t k = canon_key(src, dst, s->symmetrize);
	return 1u + (uint32_t)(mix64(s->weight_seed ^ mix64(k)) % s->weight_max);
}

static lg_status check_spec(const lg_graph_spec* s) {
	if (!s) return set_error(LG_EINVAL, "null spec");
	if (s->scale < 1 || s->scale > 31)
		return set_error(LG_EINVAL, "scale must be in [1, 31]");
	if (!(s->edge_factor > 0) || s->a < 0 || s->b < 0 || s->c < 0
			|| s->a + s->b + s->c > 1.0 + 1e-12)
		return set_error(LG_EINVAL, "bad R-MAT parameters");
	if (s->num_levels < 1 || s->num_levels > LG_MAX_LEVELS)
		return set_error(LG_EINVAL, "bad number of levels");
	if (!(s->level0_fraction > 0 && s->level0_fraction <= 1.0))
		return set_error(LG_EINVAL, "level0_fraction must be in (0, 1]");
	if (s->delete_fraction < 0 || s->delete_fraction >= 1)
		return set_error(LG_EINVAL, "delete_fraction must be in [0, 1)");
	return LG_OK;
}

lg_status lg_gen_edges(const lg_graph_spec* s, uint32_t* src, uint32_t* dst,
		uint64_t capacity, uint64_t* n) {
	clear_error();
	lg_status st = check_spec(s);
	if (st) return st;
	if (!src || !dst || !n) return set_error(LG_EINVAL, "null output");
	uint64_t V = 1ull << s->scale;
	uint64_t draws = (uint64_t)llround(s->edge_factor * (double)V);
	uint64_t need = s->symmetrize ? 2 * draws : draws;
	if (capacity < need) return set_error(LG_EINVAL, "capacity too small");
	try {
		std::vector<uint64_t> keys(need);
		double a = s->a, ab = s->a + s->b, abc = s->a + s->b + s->c;
		const uint64_t SKIP = ~0ull;
#pragma omp parallel for schedule(static)
		for (uint64_t i = 0; i < draws; i++) {
			uint32_t u, v;
			rmat_draw(s->seed, i, s->scale, a, ab, abc, &u, &v);
			if (s->kind == LG_GEN_KRONECKER) {
				u = scramble_id(u, s->scale, s->seed);
				v = scramble_id(v, s->scale, s->seed);
			}
			if (u == v) {
				keys[i] = SKIP;
				if (s->symmetrize) keys[draws + i] = SKIP;
			} else {
				keys[i] = ((uint64_t)u << 32) | v;
				if (s->symmetrize) keys[draws + i] = ((uint64_t)v << 32) | u;
			}
		}
		radix_sort_u64(keys, nullptr);
		uint64_t m = 0;
		for (uint64_t i = 0; i < need; i++) {
			if (keys[i] == SKIP) break;
			if (m > 0 && keys[i] == keys[m - 1]) continue;
			keys[m++] = keys[i];
		}
#pragma omp parallel for
		for (uint64_t i = 0; i < m; i++) {
			src[i] = (uint32_t)(keys[i] >> 32);
			dst[i] = (uint32_t)keys[i];
		}
		*n = m;
	} catch (const std::bad_alloc&) {
		return set_error(LG_ENOMEM, "out of host memory generating edges");
	}
	return LG_OK;
}

lg_status lg_hgraph_build(lg_hgraph* g, const lg_graph_spec* s) {
	clear_error();
	lg_status st = check_spec(s);
	if (st) return st;
	if (!g) return set_error(LG_EINVAL, "null graph");
	if (g->V != (1ull << s->scale))
		return set_error(LG_EINVAL, "graph size differs from 2^scale");
	if (!g->out.vt.empty()) return set_error(LG_ESTATE, "graph is not empty");
	try {
		uint64_t V = 1ull << s->scale;
		uint64_t draws = (uint64_t)llround(s->edge_factor * (double)V);
		uint64_t cap = s->symmetrize ? 2 * draws : draws;
		std::vector<uint32_t> src(cap), dst(cap);
		uint64_t n = 0;
		st = lg_gen_edges(s, src.data(), dst.data(), cap, &n);
		if (st) return st;
		const int L = s->num_levels;
		const double f0 = s->level0_fraction, p = s->delete_fraction;
		// Level of insertion and of deletion of every edge, decided on the
		// canonical (unordered when symmetric) pair so both arcs agree.
		std::vector<uint8_t> lev_add(n), lev_del(n);
#pragma omp parallel for schedule(static)
		for (uint64_t i = 0; i < n; i++) {
			uint64_t k = canon_key(src[i], dst[i], s->symmetrize);
			double u = unit_double(mix64(s->split_seed ^ mix64(k)));
			int la = 0;
			if (L > 1 && u >= f0) {
				la = 1 + (int)((u - f0) / (1.0 - f0) * (double)(L - 1));
				if (la > L - 1) la = L - 1;
			}
			int ld = 255;
			for (int l = la + 1; l < L && p > 0; l++) {
				double r = unit_double(mix64(mix64(s->split_seed + 0x51ed27u * (uint64_t)l) ^ k));
				if (r < p) { ld = l; break; }
			}
			lev_add[i] = (uint8_t)la;
			lev_del[i] = (uint8_t)ld;
		}
		for (int l = 0; l < L; l++) {
			std::vector<uint32_t> ns, nd, ds, dd, w;
			uint64_t cn = 0, cd = 0;
#pragma omp parallel for reduction(+:cn, cd)
			for (uint64_t i = 0; i < n; i++) {
				cn += lev_add[i] == l;
				cd += lev_del[i] == l;
			}
			ns.resize(cn); nd.resize(cn); ds.resize(cd); dd.resize(cd);
			if (s->weight_max) w.resize(cn);
			// order-preserving parallel compaction
			int nt = omp_get_max_threads();
			std::vector<uint64_t> pa(nt + 1, 0), pd(nt + 1, 0);
#pragma omp parallel num_threads(nt)
			{
				int t = omp_get_thread_num();
				uint64_t lo = n * t / nt, hi = n * (t + 1) / nt, a = 0, d = 0;
				for (uint64_t i = lo; i < hi; i++) {
					a += lev_add[i] == l; d += lev_del[i] == l;
				}
				pa[t + 1] = a; pd[t + 1] = d;
#pragma omp barrier
#pragma omp single
				for (int k = 0; k < nt; k++) { pa[k + 1] += pa[k]; pd[k + 1] += pd[k]; }
				uint64_t ia = pa[t], id = pd[t];
				for (uint64_t i = lo; i < hi; i++) {
					if (lev_add[i] == l) {
						ns[ia] = src[i]; nd[ia] = dst[i];
						if (s->weight_max) w[ia] = lg_gen_weight(s, src[i], dst[i]);
						ia++;
					}
					if (lev_del[i] == l) { ds[id] = src[i]; dd[id] = dst[i]; id++; }
				}
			}
			st = lg_hgraph_add_level(g, ns.data(), nd.data(), cn, ds.data(),
					dd.data(), cd, s->weight_max ? w.data() : nullptr);
			if (st) return st;
		}
	} catch (const std::bad_alloc&) {
		return set_error(LG_ENOMEM, "out of host memory building the graph");
	}
	return LG_OK;
}

} // extern "C"
