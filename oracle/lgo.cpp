// lgo.cpp - CPU ORACLE for the LLAMA analytics path.
//
// TEST INFRASTRUCTURE ONLY.  This file restates, serially and plainly, the
// reference's multiversioned CSR and its benchmark kernels so that the CUDA
// engine (llama_b200/) can be checked against it.  Only tests/, the smoke
// check and the CPU-baseline leg of bench.py may load it; the product never
// does.  It is itself pinned against the reference code compiled from source
// (oracle/ref_harness.cc -> oracle/_ref/) and against the committed golden
// fixtures in tests/golden/.
//
// Every function names the reference lines it restates (paths relative to
// the goatdb/llama source tree).

#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <cmath>
#include <limits>
#include <queue>
#include <vector>

namespace {

const int BITS_LEVEL = 26;                          // ll_mlcsr_helpers.h:62
const int BITS_INDEX = 64 - BITS_LEVEL;             // ll_mlcsr_helpers.h:68
const int64_t NIL = -1;                             // ll_common.h:118-120
const uint64_t FRESH = (1ull << BITS_LEVEL) - 1;    // LL_MAX_LEVEL + 2, :102
const int32_t UNREACHED = 2147483646;               // INT_MAX - 1, sssp.h:108

inline int64_t edge_create(uint64_t level, uint64_t index) {   // :76
	return (int64_t)((level << BITS_INDEX) | index);
}
inline uint64_t edge_level(int64_t e) { return (uint64_t)e >> BITS_INDEX; }       // :77
inline uint64_t edge_index(int64_t e) { return (uint64_t)e & ((1ull << BITS_INDEX) - 1); } // :78
inline uint64_t value_create_ext(uint64_t payload, uint64_t maxlev) {  // :98-101
	return payload | (maxlev << BITS_INDEX);
}
inline uint64_t value_payload(uint64_t x) { return x & ((1ull << BITS_INDEX) - 1); } // :104
inline uint64_t value_max_level(uint64_t x) { return x >> BITS_INDEX; }              // :105
inline bool value_is_deleted(uint64_t x, uint64_t level) {                           // :107
	return value_max_level(x) <= level;
}

struct VtEntry {            // ll_mlcsr_core__begin_t, ll_mlcsr_helpers.h:141-149
	int64_t adj_list_start;
	uint32_t level_length;
	uint32_t degree;
};

struct Csr {
	std::vector<std::vector<VtEntry>> vt;     // per level, max_nodes + 1
	std::vector<std::vector<uint64_t>> et;    // per level edge table
	std::vector<std::vector<uint32_t>> w;     // per level edge property
	uint64_t min_level = 0;                   // _minLevel, ll_mlcsr_sp.h:114-116
};

struct Iter {               // ll_edge_iterator, ll_mlcsr_iterator.h:53-68
	int64_t edge;
	uint64_t left;
	uint64_t ptr_level, ptr_index;
	int64_t node;
	int64_t last_node;
	uint64_t max_level;
};

// iter_descend, ll_mlcsr_sp.h:2090-2134: the continuation record is the
// 16 bytes right after the last slot of the fragment.
void iter_descend(const Csr& c, Iter& it) {
	uint64_t level = edge_level(it.edge);
	if (level == 0 || (uint64_t)it.node >= c.vt[level - 1].size() - 1) {
		it.edge = NIL;
		return;
	}
	VtEntry b;
	memcpy(&b, &c.et[it.ptr_level][it.ptr_index + 1], sizeof(b));
	it.edge = b.adj_list_start;
	if (edge_level(it.edge) < c.min_level) {      // LL_MIN_LEVEL, :2107-2110
		it.left = 0;
		it.edge = NIL;
		return;
	}
	it.left = b.level_length;
	if (it.left == 0) it.edge = NIL;
	else { it.ptr_level = edge_level(it.edge); it.ptr_index = edge_index(it.edge); }
}

// is_edge_deleted, ll_mlcsr_sp.h:1290-1310
bool is_deleted(const Csr& c, const Iter& it) {
	if (it.edge == NIL) return false;
	uint64_t v = c.et[edge_level(it.edge)][edge_index(it.edge)];
	return value_is_deleted(v, it.max_level);
}

// iter_next, ll_mlcsr_sp.h:2145-2196
int64_t iter_next(const Csr& c, Iter& it) {
	int64_t r = it.edge;
	if (r != NIL) {
		it.last_node = (int64_t)value_payload(c.et[it.ptr_level][it.ptr_index]);
		do {
			if (it.left > 1) {
				it.left--;
				it.edge = it.edge + 1;
				it.ptr_index++;
			} else {
				iter_descend(c, it);
			}
		} while (is_deleted(c, it));
	}
	return r;
}

// iter_begin, ll_mlcsr_sp.h:1994-2053 (level = snapshot, max_level = level)
void iter_begin(const Csr& c, Iter& it, int64_t n, int level) {
	it.node = n;
	it.max_level = level;
	const VtEntry& b = c.vt[level][n];
	it.edge = b.adj_list_start;
	if (edge_level(it.edge) < c.min_level) {      // LL_MIN_LEVEL, :2021-2026
		it.left = 0;
		it.edge = NIL;
		return;
	}
	it.left = b.level_length;
	if (it.left == 0) it.edge = NIL;
	else { it.ptr_level = edge_level(it.edge); it.ptr_index = edge_index(it.edge); }
	if (is_deleted(c, it)) {
		int64_t keep = it.last_node;
		iter_next(c, it);
		it.last_node = keep;
	}
}

// Neighbours in iteration order (ll_foreach_out / ll_foreach_in,
// ll_mlcsr_iterator.h:186-214), with the edge id of each.
void neighbours(const Csr& c, int level, int64_t n, std::vector<uint32_t>& nb,
		std::vector<int64_t>* ids) {
	nb.clear();
	if (ids) ids->clear();
	Iter it;
	it.last_node = -1;
	iter_begin(c, it, n, level);
	for (int64_t e = iter_next(c, it); e != NIL; e = iter_next(c, it)) {
		nb.push_back((uint32_t)it.last_node);
		if (ids) ids->push_back(e);
	}
}

// degree(n): the vertex-table degree (LL_PRECOMPUTED_DEGREE,
// ll_mlcsr_sp.h:1900-1930).  In a sliding window it is the number of edges
// the iterator yields: the reference leaves the windowed degree with
// deletions unimplemented (ll_mlcsr_sp.h:1914-1928).
std::vector<uint32_t> degrees_of(const Csr& c, int level, uint64_t V) {
	std::vector<uint32_t> d(V);
	std::vector<uint32_t> nb;
	for (uint64_t v = 0; v < V; v++) {
		if (c.min_level == 0) { d[v] = c.vt[level][v].degree; continue; }
		neighbours(c, level, (int64_t)v, nb, nullptr);
		d[v] = (uint32_t)nb.size();
	}
	return d;
}

// find, ll_mlcsr_sp.h:2334-2356: first edge of n whose payload is `value`.
int64_t find_edge(const Csr& c, int level, int64_t n, uint64_t value) {
	Iter it;
	it.last_node = -1;
	iter_begin(c, it, n, level);
	for (int64_t e = iter_next(c, it); e != NIL; e = iter_next(c, it))
		if ((uint64_t)it.last_node == value) return e;
	return NIL;
}

// One level of one CSR: init_level_from_degrees (ll_mlcsr_sp.h:1562-1607)
// -> init_node per vertex (:1375-1550) -> finish_level_vertices (:786-808),
// then write_value for every new edge (:1618-1627), fragments sorted by
// target.  `adj[v]` are the new neighbours of v (sorted), `del[v]` the number
// of v's edges this level deletes.
void build_level(Csr& c, uint64_t V, const std::vector<std::vector<uint32_t>>& adj,
		const std::vector<uint32_t>& del, const std::vector<std::vector<uint32_t>>* wts) {
	const int level = (int)c.vt.size();
	std::vector<VtEntry> vt;
	uint64_t prev_size = 0;
	if (level > 0) {
		vt = c.vt[level - 1];                     // copy-on-write: start shared
		prev_size = vt.size() - 1;
		VtEntry zero = {0, 0, 0};
		vt.resize(V + 1, zero);
	} else {
		VtEntry nil = {NIL, 0, 0};
		vt.assign(V + 1, nil);
	}
	const std::vector<VtEntry>* prev = level > 0 ? &c.vt[level - 1] : nullptr;
	std::vector<uint64_t> et;
	std::vector<uint32_t> wt;
	uint64_t write_index = 0;
	std::vector<uint64_t> start(V, 0);
	for (uint64_t node = 0; node < V; node++) {
		uint64_t new_edges = adj[node].size();
		uint64_t deleted = level == 0 ? 0 : del[node];
		VtEntry e = {0, 0, 0};
		if (!(level == 0 || new_edges > 0 || deleted > 0)) {
			if (node >= prev_size) { e.adj_list_start = NIL; vt[node] = e; }
			continue;
		}
		if (level == 0 || new_edges > 0) {
			e.adj_list_start = new_edges == 0 ? NIL : edge_create(level, write_index);
			e.level_length = (uint32_t)new_edges;
		} else {
			if (node >= prev_size) e.adj_list_start = NIL;
			else e = (*prev)[node];
		}
		e.degree = (uint32_t)(new_edges - deleted);
		if (level > 0 && node < prev_size) {
			const VtEntry& bprev = (*prev)[node];
			if (bprev.adj_list_start != NIL) e.degree = e.degree + bprev.degree;
		}
		if (e.degree == 0) { e.adj_list_start = NIL; e.level_length = 0; }
		uint64_t delta = new_edges;
		start[node] = write_index;
		if (level > 0 && e.adj_list_start != NIL) {
			uint64_t t = write_index + new_edges;
			VtEntry x = {NIL, 0, 0};
			if (node < prev_size) x = (*prev)[node];
			if (et.size() < t + 2) { et.resize(t + 2, 0); wt.resize(t + 2, 0); }
			memcpy(&et[t], &x, sizeof(x));
			delta += 2;
		}
		vt[node] = e;
		write_index += delta;
	}
	VtEntry sentinel = {edge_create(level, write_index), 0, 0};
	vt[V] = sentinel;
	et.resize(write_index, 0);
	wt.resize(write_index, 0);
	for (uint64_t node = 0; node < V; node++)
		for (uint64_t k = 0; k < adj[node].size(); k++) {
			et[start[node] + k] = value_create_ext(adj[node][k], FRESH);
			if (wts) wt[start[node] + k] = (*wts)[node][k];
		}
	c.vt.push_back(std::move(vt));
	c.et.push_back(std::move(et));
	c.w.push_back(std::move(wt));
}

struct Graph {
	uint64_t V;
	Csr out, in;
};

} // namespace

extern "C" {

void* lgo_create(uint64_t V) {
	Graph* g = new Graph();
	g->V = V;
	return g;
}

void lgo_destroy(void* g) { delete (Graph*)g; }

int lgo_num_levels(void* gp) { return (int)((Graph*)gp)->out.vt.size(); }

// Sliding window: ll_mlcsr_ro_graph::set_min_level (ll_mlcsr_graph.h:560-602)
// on both CSRs.
void lgo_set_min_level(void* gp, int m) {
	Graph* g = (Graph*)gp;
	g->out.min_level = (uint64_t)m;
	g->in.min_level = (uint64_t)m;
}

// Append a level: new edges (any order), deleted edges (live in the latest
// snapshot), optional weights per new edge.  Deletions lower the slot's
// max_visible_level to the new level number in both CSRs
// (update_max_visible_level_lower_only, ll_mlcsr_sp.h:849-863, as called
// from ll_writable_graph.h:936-945).  Returns 0 or -1 on bad input.
int lgo_add_level(void* gp, const uint32_t* src, const uint32_t* dst, uint64_t n,
		const uint32_t* dsrc, const uint32_t* ddst, uint64_t nd,
		const uint32_t* weights) {
	Graph* g = (Graph*)gp;
	const uint64_t V = g->V;
	const int level = (int)g->out.vt.size();
	std::vector<std::vector<uint32_t>> oadj(V), iadj(V), ow(V);
	std::vector<std::pair<std::pair<uint32_t, uint32_t>, uint32_t>> e(n);
	for (uint64_t i = 0; i < n; i++) {
		if (src[i] >= V || dst[i] >= V) return -1;
		e[i] = {{src[i], dst[i]}, weights ? weights[i] : 0u};
	}
	std::sort(e.begin(), e.end());
	for (uint64_t i = 0; i < n; i++) {
		oadj[e[i].first.first].push_back(e[i].first.second);
		ow[e[i].first.first].push_back(e[i].second);
	}
	for (uint64_t i = 0; i < n; i++) iadj[e[i].first.second].push_back(e[i].first.first);
	std::vector<uint32_t> odel(V, 0), idel(V, 0);
	std::vector<int64_t> oe(nd), ie(nd);
	for (uint64_t i = 0; i < nd; i++) {
		if (level == 0) return -1;
		oe[i] = find_edge(g->out, level - 1, dsrc[i], ddst[i]);
		ie[i] = find_edge(g->in, level - 1, ddst[i], dsrc[i]);
		if (oe[i] == NIL || ie[i] == NIL) return -1;
		odel[dsrc[i]]++;
		idel[ddst[i]]++;
	}
	build_level(g->out, V, oadj, odel, weights ? &ow : nullptr);
	build_level(g->in, V, iadj, idel, nullptr);
	for (uint64_t i = 0; i < nd; i++) {
		for (int d = 0; d < 2; d++) {
			Csr& c = d == 0 ? g->out : g->in;
			int64_t x = d == 0 ? oe[i] : ie[i];
			uint64_t& v = c.et[edge_level(x)][edge_index(x)];
			if ((uint64_t)level < value_max_level(v))
				v = value_create_ext(value_payload(v), (uint64_t)level);
		}
	}
	return 0;
}

// Level arrays, for byte comparison with other builders.
int lgo_level_arrays(void* gp, int dir, int level, const void** vt,
		uint64_t* n_vt, const uint64_t** et, uint64_t* n_et) {
	Graph* g = (Graph*)gp;
	Csr& c = dir == 0 ? g->out : g->in;
	if (level < 0 || level >= (int)c.vt.size()) return -1;
	*vt = c.vt[level].data();
	*n_vt = c.vt[level].size();
	*et = c.et[level].data();
	*n_et = c.et[level].size();
	return 0;
}

// Adjacency of snapshot `level` in iteration order.  offsets: V+1 entries;
// nbr / ids may be NULL (then only offsets are written).  Returns #edges.
uint64_t lgo_adjacency(void* gp, int dir, int level, uint64_t* offsets,
		uint32_t* nbr, int64_t* ids) {
	Graph* g = (Graph*)gp;
	Csr& c = dir == 0 ? g->out : g->in;
	std::vector<uint32_t> nb;
	std::vector<int64_t> id;
	uint64_t o = 0;
	for (uint64_t v = 0; v < g->V; v++) {
		offsets[v] = o;
		neighbours(c, level, v, nb, &id);
		for (size_t k = 0; k < nb.size(); k++, o++) {
			if (nbr) nbr[o] = nb[k];
			if (ids) ids[o] = id[k];
		}
	}
	offsets[g->V] = o;
	return o;
}

// Out-degree (dir 0) or in-degree (dir 1): degree(n) with
// LL_PRECOMPUTED_DEGREE, ll_mlcsr_sp.h:1900-1930.
void lgo_degrees(void* gp, int dir, int level, uint32_t* deg) {
	Graph* g = (Graph*)gp;
	Csr& c = dir == 0 ? g->out : g->in;
	std::vector<uint32_t> d = degrees_of(c, level, g->V);
	for (uint64_t v = 0; v < g->V; v++) deg[v] = d[v];
}

// PageRank pull, FP64: ll_b_pagerank_pull_ext::run, pagerank.h:98-182.
void lgo_pagerank_pull(void* gp, int level, int max, double d, double* rank) {
	Graph* g = (Graph*)gp;
	const uint64_t V = g->V;
	const double N = (double)V;
	std::vector<double> nxt(V);
	for (uint64_t t = 0; t < V; t++) rank[t] = 1 / N;
	std::vector<uint32_t> nb;
	const std::vector<uint32_t> od = degrees_of(g->out, level, V);
	int cnt = 0;
	do {
		for (uint64_t t = 0; t < V; t++) {
			double S = 0.0;
			neighbours(g->in, level, t, nb, nullptr);
			for (uint32_t w : nb)
				S = S + rank[w] / ((double)od[w]);
			nxt[t] = (1 - d) / N + d * S;
		}
		for (uint64_t t = 0; t < V; t++) rank[t] = nxt[t];
		cnt = cnt + 1;
	} while (cnt < max);
}

// PageRank push, FP64: ll_b_pagerank_push_ext::run, pagerank.h:258-318.
// Sequential here: vertices in id order, out-edges in iteration order (the
// reference adds with an atomic in whatever order its threads run).
void lgo_pagerank_push(void* gp, int level, int max, double d, double* rank) {
	Graph* g = (Graph*)gp;
	const uint64_t V = g->V;
	const double N = (double)V;
	std::vector<double> nxt(V, 0.0);
	for (uint64_t t = 0; t < V; t++) rank[t] = 1 / N;
	std::vector<uint32_t> nb;
	const std::vector<uint32_t> od = degrees_of(g->out, level, V);
	int cnt = 0;
	do {
		for (uint64_t t = 0; t < V; t++) {
			if (od[t] == 0) continue;
			const double delta = rank[t] / od[t];
			neighbours(g->out, level, t, nb, nullptr);
			for (uint32_t w : nb) nxt[w] += delta;
		}
		for (uint64_t t = 0; t < V; t++) {
			rank[t] = (1 - d) / N + d * nxt[t];
			nxt[t] = 0.0;
		}
		cnt = cnt + 1;
	} while (cnt < max);
}

// Average teen count: ll_b_avg_teen_cnt::run, avg_teen_cnt.h:96-139.  For
// every vertex n, teen_cnt[n] = in-neighbours t with 10 <= age[t] < 20; over
// the vertices with age[n] > K, sum the counts (int32 in the reference; here
// int64, equal while the sum fits 31 bits) and return (float)(sum / count),
// 0 when no vertex qualifies.
double lgo_avg_teen_cnt(void* gp, int level, const int32_t* age, int K,
		int32_t* teen_cnt, int64_t* sum_out, int64_t* cnt_out) {
	Graph* g = (Graph*)gp;
	std::vector<uint32_t> nb;
	int64_t S = 0, cnt = 0;
	for (uint64_t n = 0; n < g->V; n++) {
		int32_t c = 0;
		neighbours(g->in, level, n, nb, nullptr);
		for (uint32_t t : nb)
			if (age[t] >= 10 && age[t] < 20) c = c + 1;
		teen_cnt[n] = c;
		if (age[n] > K) { S += c; cnt += 1; }
	}
	*sum_out = S;
	*cnt_out = cnt;
	const double avg = (0 == cnt) ? 0.0 : ((double)S / (double)cnt);
	return (double)(float)avg;
}

// BFS levels: u_sssp_bfs (sssp.h:219-244) / ll_b_sssp_unweighted_bfs::run
// (sssp.h:285-300): dist = INT_MAX-1, dist[root] = 0, level-synchronous BFS
// over out-edges.  Returns the number of reached vertices.
uint64_t lgo_bfs(void* gp, int level, int64_t root, int32_t* dist) {
	Graph* g = (Graph*)gp;
	for (uint64_t v = 0; v < g->V; v++) dist[v] = UNREACHED;
	dist[root] = 0;
	std::vector<uint32_t> frontier(1, (uint32_t)root), next, nb;
	uint64_t reached = 1;
	int32_t cur = 0;
	while (!frontier.empty()) {
		next.clear();
		for (uint32_t u : frontier) {
			neighbours(g->out, level, u, nb, nullptr);
			for (uint32_t v : nb)
				if (dist[v] == UNREACHED) { dist[v] = cur + 1; next.push_back(v); }
		}
		reached += next.size();
		frontier.swap(next);
		cur++;
	}
	return reached;
}

// Brandes betweenness centrality from explicit sources, FP64 restatement of
// bc_random_bfs (bc_random.h:55-111) over ll_bfs_template's level-synchronous
// BFS: sigma is pushed along down edges (level[w] == level[v] + 1, the edges
// is_down_edge marks, ll_bfs_template.h:337-351); the reverse sweep visits
// levels deepest first and sets delta[v] = sum over down edges v->w of
// sigma[v] / sigma[w] * (1 + delta[w]), then BC[v] += delta[v] for v != s.
void lgo_bc(void* gp, int level, const int64_t* sources, int n, double* bc) {
	Graph* g = (Graph*)gp;
	const uint64_t V = g->V;
	std::vector<int32_t> lev(V);
	std::vector<double> sigma(V), delta(V);
	std::vector<uint32_t> nb;
	for (uint64_t v = 0; v < V; v++) bc[v] = 0.0;
	for (int i = 0; i < n; i++) {
		const int64_t s = sources[i];
		std::fill(lev.begin(), lev.end(), -1);
		std::fill(sigma.begin(), sigma.end(), 0.0);
		std::vector<std::vector<uint32_t>> levels(1, std::vector<uint32_t>(1, (uint32_t)s));
		lev[s] = 0;
		sigma[s] = 1.0;
		for (int32_t cur = 0; !levels[cur].empty(); cur++) {
			levels.emplace_back();
			for (uint32_t v : levels[cur]) {
				neighbours(g->out, level, v, nb, nullptr);
				for (uint32_t w : nb)
					if (lev[w] < 0) { lev[w] = cur + 1; levels[cur + 1].push_back(w); }
			}
			for (uint32_t v : levels[cur]) {          // visit_fw
				neighbours(g->out, level, v, nb, nullptr);
				for (uint32_t w : nb)
					if (lev[w] == cur + 1) sigma[w] += sigma[v];
			}
		}
		for (int32_t cur = (int32_t)levels.size() - 1; cur >= 0; cur--) {   // visit_rv
			for (uint32_t v : levels[cur]) {
				if ((int64_t)v == s) continue;
				double S = 0.0;
				neighbours(g->out, level, v, nb, nullptr);
				for (uint32_t w : nb)
					if (lev[w] == cur + 1) S = S + sigma[v] / sigma[w] * (1 + delta[w]);
				delta[v] = S;
				bc[v] = bc[v] + delta[v];
			}
		}
	}
}

// Weighted SSSP: ll_b_sssp_weighted::run (sssp.h:97-183), frontier
// Bellman-Ford to a fixpoint with G_len[e] = the per-slot edge property
// (ll_mlcsr_properties.h:985-1005).  dist = INT_MAX-1 when unreached.
// Returns the number of reached vertices (the finalize() value).
uint64_t lgo_sssp(void* gp, int level, int64_t root, uint32_t* dist_out) {
	Graph* g = (Graph*)gp;
	const uint64_t V = g->V;
	const uint64_t INF = UNREACHED;
	std::vector<uint64_t> dist(V, INF), nxt(V, INF);
	std::vector<char> upd(V, 0), upd_n(V, 0);
	dist[root] = nxt[root] = 0;
	upd[root] = 1;
	std::vector<uint32_t> nb;
	std::vector<int64_t> ids;
	bool fin = false;
	while (!fin) {
		for (uint64_t n = 0; n < V; n++) {
			if (!upd[n]) continue;
			neighbours(g->out, level, n, nb, &ids);
			for (size_t k = 0; k < nb.size(); k++) {
				uint64_t w = g->out.w[edge_level(ids[k])][edge_index(ids[k])];
				uint64_t cand = dist[n] + w;
				if (nxt[nb[k]] > cand) { nxt[nb[k]] = cand; upd_n[nb[k]] = 1; }
			}
		}
		bool any = false;
		for (uint64_t t = 0; t < V; t++) {
			dist[t] = nxt[t];
			upd[t] = upd_n[t];
			upd_n[t] = 0;
			any = any || upd[t];
		}
		fin = !any;
	}
	uint64_t count = 0;
	for (uint64_t v = 0; v < V; v++) {
		dist_out[v] = (uint32_t)dist[v];
		count += dist[v] < INF;
	}
	return count;
}

// Triangle counting on the symmetrised, de-duplicated snapshot (what tc_u
// computes on a graph loaded with -U and flattened to one level,
// triangle_counting.h:343-470): triangles u < v < w with all three
// undirected edges present, each counted once.
int64_t lgo_tc(void* gp, int level) {
	Graph* g = (Graph*)gp;
	const uint64_t V = g->V;
	std::vector<std::vector<uint32_t>> adj(V);
	std::vector<uint32_t> nb;
	for (uint64_t v = 0; v < V; v++) {
		neighbours(g->out, level, v, nb, nullptr);
		for (uint32_t w : nb)
			if (w != v) { adj[v].push_back(w); adj[w].push_back((uint32_t)v); }
	}
	for (auto& a : adj) {
		std::sort(a.begin(), a.end());
		a.erase(std::unique(a.begin(), a.end()), a.end());
	}
	int64_t T = 0;
	for (uint64_t u = 0; u < V; u++)
		for (uint32_t v : adj[u]) {
			if (v <= u) continue;
			// count_for: common neighbours of u and v greater than v
			size_t i = 0, j = 0;
			const auto &A = adj[u], &B = adj[v];
			while (i < A.size() && j < B.size()) {
				if (A[i] < B[j]) i++;
				else if (B[j] < A[i]) j++;
				else { if (A[i] > v) T++; i++; j++; }
			}
		}
	return T;
}

// Strongly connected components of the snapshot, labelled by the smallest
// vertex id of each component.  The reference's tarjan_scc
// (tarjan_scc.h:55-206) uses vertex ids as low-links and does not compute
// true SCCs, so this is a plain iterative Tarjan with discovery indices.
void lgo_scc(void* gp, int level, int64_t* label) {
	Graph* g = (Graph*)gp;
	const uint64_t V = g->V;
	std::vector<std::vector<uint32_t>> adj(V);
	for (uint64_t v = 0; v < V; v++) neighbours(g->out, level, v, adj[v], nullptr);
	std::vector<int64_t> idx(V, -1), low(V, 0);
	std::vector<char> on(V, 0);
	std::vector<uint32_t> stk;
	std::vector<std::pair<uint32_t, size_t>> call;
	int64_t counter = 0;
	for (uint64_t r = 0; r < V; r++) {
		if (idx[r] >= 0) continue;
		call.push_back({(uint32_t)r, 0});
		idx[r] = low[r] = counter++;
		stk.push_back((uint32_t)r);
		on[r] = 1;
		while (!call.empty()) {
			uint32_t v = call.back().first;
			size_t& k = call.back().second;
			if (k < adj[v].size()) {
				uint32_t w = adj[v][k++];
				if (idx[w] < 0) {
					idx[w] = low[w] = counter++;
					stk.push_back(w);
					on[w] = 1;
					call.push_back({w, 0});
				} else if (on[w]) {
					low[v] = std::min(low[v], idx[w]);
				}
			} else {
				if (low[v] == idx[v]) {
					std::vector<uint32_t> comp;
					uint32_t w;
					do { w = stk.back(); stk.pop_back(); on[w] = 0; comp.push_back(w); }
					while (w != v);
					int64_t m = *std::min_element(comp.begin(), comp.end());
					for (uint32_t x : comp) label[x] = m;
				}
				call.pop_back();
				if (!call.empty()) {
					uint32_t p = call.back().first;
					low[p] = std::min(low[p], low[v]);
				}
			}
		}
	}
}

// Weighted PageRank to a fixed point (no reference counterpart; the pull
// iteration of pagerank.h:120-169 with per-edge weights and a teleport
// vector): x' = (1-d) v + d P^T x, P(w->t) = weight of the out-edge, given in
// the snapshot's out-adjacency iteration order.  Starts at x = v, stops when
// sum |x' - x| < tol.  Returns the number of iterations.
int lgo_wpr_forward(void* gp, int level, const double* w, const double* v, double d,
		double tol, int max_iter, double* x) {
	Graph* g = (Graph*)gp;
	const uint64_t V = g->V;
	std::vector<std::vector<uint32_t>> out(V);
	for (uint64_t u = 0; u < V; u++) neighbours(g->out, level, u, out[u], nullptr);
	std::vector<double> nx(V);
	for (uint64_t t = 0; t < V; t++) x[t] = v[t];
	int it = 0;
	while (it < max_iter) {
		for (uint64_t t = 0; t < V; t++) nx[t] = (1 - d) * v[t];
		uint64_t p = 0;
		for (uint64_t u = 0; u < V; u++)
			for (uint32_t t : out[u]) nx[t] += d * (w[p++] * x[u]);
		double r = 0;
		for (uint64_t t = 0; t < V; t++) { r += std::fabs(nx[t] - x[t]); x[t] = nx[t]; }
		it++;
		if (r < tol) break;
	}
	return it;
}

// Adjoint of lgo_wpr_forward by implicit differentiation: with
// g = dL/dx, lambda solves lambda = g + d P lambda (the transposed fixed
// point, iterated over out-edges), and dL/dv = (1-d) lambda,
// dL/dP(w->t) = d lambda[t] x[w].  Returns the number of iterations.
int lgo_wpr_backward(void* gp, int level, const double* w, const double* x,
		const double* gv, double d, double tol, int max_iter, double* dldw,
		double* dldv) {
	Graph* g = (Graph*)gp;
	const uint64_t V = g->V;
	std::vector<std::vector<uint32_t>> out(V);
	for (uint64_t u = 0; u < V; u++) neighbours(g->out, level, u, out[u], nullptr);
	std::vector<double> lam(gv, gv + V), nl(V);
	int it = 0;
	while (it < max_iter) {
		uint64_t p = 0;
		double r = 0;
		for (uint64_t u = 0; u < V; u++) {
			double s = 0;
			for (uint32_t t : out[u]) s += w[p++] * lam[t];
			nl[u] = gv[u] + d * s;
		}
		for (uint64_t u = 0; u < V; u++) { r += std::fabs(nl[u] - lam[u]); lam[u] = nl[u]; }
		it++;
		if (r < tol) break;
	}
	uint64_t p = 0;
	for (uint64_t u = 0; u < V; u++)
		for (uint32_t t : out[u]) dldw[p++] = d * lam[t] * x[u];
	for (uint64_t t = 0; t < V; t++) dldv[t] = (1 - d) * lam[t];
	return it;
}

// Personalized PageRank with K single-vertex teleport seeds, the pull
// iteration of pagerank.h:120-169 with the uniform teleport (1-d)/N replaced
// by (1-d) * [t == seed_k]: x0 = e_seed, then `iters` times
// x'[t] = (1-d) [t == seed] + d * sum_{w in in(t)} x[w] / out_degree(w).
// out is vertex-major: out[v * K + k].
void lgo_ppr(void* gp, int level, const int64_t* seeds, int K, int iters,
		double d, double* out) {
	Graph* g = (Graph*)gp;
	const uint64_t V = g->V;
	std::vector<double> x(V), nx(V);
	std::vector<uint32_t> nb;
	std::vector<std::vector<uint32_t>> in(V);
	for (uint64_t t = 0; t < V; t++) neighbours(g->in, level, t, in[t], nullptr);
	const std::vector<uint32_t> od = degrees_of(g->out, level, V);
	for (int k = 0; k < K; k++) {
		std::fill(x.begin(), x.end(), 0.0);
		x[seeds[k]] = 1.0;
		for (int it = 0; it < iters; it++) {
			for (uint64_t t = 0; t < V; t++) {
				double S = 0.0;
				for (uint32_t w : in[t])
					S = S + x[w] / ((double)od[w]);
				nx[t] = ((int64_t)t == seeds[k] ? (1 - d) : 0.0) + d * S;
			}
			x.swap(nx);
		}
		for (uint64_t v = 0; v < V; v++) out[v * K + k] = x[v];
	}
}

} // extern "C"

// ---------------------------------------------------------------------------
// At-size checks.  The functions below work on plain CSR arrays (offsets +
// neighbour ids), such as the adjacency the reference's own iterator returns
// for a snapshot (oracle/_ref), and use OpenMP so that the benchmark's
// full-size workloads can be checked on the host cores in seconds.  Each is
// pinned against the serial store-walking function above on small graphs
// (tests/test_oracle_at_size.py).
// ---------------------------------------------------------------------------

#include <omp.h>
#include <parallel/algorithm>

namespace {

inline uint64_t gen_mix64(uint64_t z) {            // splitmix64 finaliser
	z += 0x9e3779b97f4a7c15ull;
	z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
	z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
	return z ^ (z >> 31);
}
inline double gen_unit(uint64_t h) { return (double)(h >> 11) * (1.0 / 9007199254740992.0); }
inline uint64_t gen_canon(uint32_t s, uint32_t t, int symmetric) {
	if (symmetric && t < s) std::swap(s, t);
	return ((uint64_t)s << 32) | t;
}
inline uint32_t gen_scramble(uint64_t x, int scale, uint64_t seed) {
	const uint64_t mask = (scale >= 64) ? ~0ull : ((1ull << scale) - 1);
	const uint64_t k1 = gen_mix64(seed ^ 0x1234567ull) | 1ull;
	const uint64_t k2 = gen_mix64(seed ^ 0x89abcdefull);
	const uint64_t k3 = gen_mix64(seed ^ 0x13579bdfull) | 1ull;
	const int half = scale / 2 > 0 ? scale / 2 : 1;
	x = (x * k1 + k2) & mask;
	x ^= x >> half;
	x = (x * k3) & mask;
	x ^= x >> half;
	x = (x * k1 + (k2 >> 7)) & mask;
	return (uint32_t)x;
}

struct GenLevel { std::vector<uint32_t> src, dst, dsrc, ddst, w; };
struct Gen { std::vector<GenLevel> lv; };

} // namespace

extern "C" {

// Parameters of a seeded workload, field for field the engine's
// lg_graph_spec (include/lg_host.h).
typedef struct lgo_gen_spec {
	int kind;                  // 0 R-MAT, 1 Kronecker (scrambled ids)
	int scale;
	double edge_factor, a, b, c;
	uint64_t seed;
	int symmetrize, num_levels;
	double level0_fraction, delete_fraction;
	uint64_t split_seed;
	uint32_t weight_max;
	uint64_t weight_seed;
} lgo_gen_spec;

// The benchmark workloads' levels, generated without the engine: R-MAT
// quadrant recursion on splitmix64 hashes of (seed, draw index), self-loops
// and duplicates dropped, every edge's insertion level and deletion level
// decided by hashes of its canonical pair, weights by a hash of the pair.
// This is the generator specification the engine's host builder
// implements (lg_hgraph_build); a CPU test checks that both produce the same
// levels.  Returns a handle, or null on bad parameters.
void* lgo_gen_create(const lgo_gen_spec* s) {
	if (!s || s->scale < 1 || s->scale > 31 || s->num_levels < 1 || s->num_levels > 64)
		return nullptr;
	const uint64_t V = 1ull << s->scale;
	const uint64_t draws = (uint64_t)llround(s->edge_factor * (double)V);
	const uint64_t need = s->symmetrize ? 2 * draws : draws;
	const double a = s->a, ab = s->a + s->b, abc = s->a + s->b + s->c;
	const uint64_t SKIP = ~0ull;
	std::vector<uint64_t> keys(need);
#pragma omp parallel for schedule(static)
	for (uint64_t i = 0; i < draws; i++) {
		uint64_t state = gen_mix64(s->seed * 0x2545f4914f6cdd1dull + i);
		uint32_t u = 0, v = 0;
		for (int k = 0; k < s->scale; k++) {
			state = gen_mix64(state);
			const double r = gen_unit(state);
			const uint32_t row = r < ab ? 0u : 1u;
			const uint32_t col = (r < a || (r >= ab && r < abc)) ? 0u : 1u;
			u = (u << 1) | row;
			v = (v << 1) | col;
		}
		if (s->kind == 1) {
			u = gen_scramble(u, s->scale, s->seed);
			v = gen_scramble(v, s->scale, s->seed);
		}
		const bool loop = u == v;
		keys[i] = loop ? SKIP : (((uint64_t)u << 32) | v);
		if (s->symmetrize) keys[draws + i] = loop ? SKIP : (((uint64_t)v << 32) | u);
	}
	__gnu_parallel::sort(keys.begin(), keys.end());
	uint64_t n = 0;
	for (uint64_t i = 0; i < need && keys[i] != SKIP; i++)
		if (n == 0 || keys[i] != keys[n - 1]) keys[n++] = keys[i];
	const int L = s->num_levels;
	const double f0 = s->level0_fraction, p = s->delete_fraction;
	std::vector<uint8_t> la(n), ld(n);
#pragma omp parallel for schedule(static)
	for (uint64_t i = 0; i < n; i++) {
		const uint32_t u = (uint32_t)(keys[i] >> 32), v = (uint32_t)keys[i];
		const uint64_t k = gen_canon(u, v, s->symmetrize);
		const double x = gen_unit(gen_mix64(s->split_seed ^ gen_mix64(k)));
		int add = 0;
		if (L > 1 && x >= f0) {
			add = 1 + (int)((x - f0) / (1.0 - f0) * (double)(L - 1));
			if (add > L - 1) add = L - 1;
		}
		int del = 255;
		for (int l = add + 1; l < L && p > 0; l++) {
			const double r = gen_unit(gen_mix64(gen_mix64(s->split_seed + 0x51ed27u * (uint64_t)l) ^ k));
			if (r < p) { del = l; break; }
		}
		la[i] = (uint8_t)add;
		ld[i] = (uint8_t)del;
	}
	Gen* g = new Gen();
	g->lv.resize(L);
	for (uint64_t i = 0; i < n; i++) {
		const uint32_t u = (uint32_t)(keys[i] >> 32), v = (uint32_t)keys[i];
		GenLevel& A = g->lv[la[i]];
		A.src.push_back(u);
		A.dst.push_back(v);
		if (s->weight_max) {
			const uint64_t k = gen_canon(u, v, s->symmetrize);
			A.w.push_back(1u + (uint32_t)(gen_mix64(s->weight_seed ^ gen_mix64(k)) % s->weight_max));
		}
		if (ld[i] != 255) { g->lv[ld[i]].dsrc.push_back(u); g->lv[ld[i]].ddst.push_back(v); }
	}
	return g;
}

void lgo_gen_destroy(void* h) { delete (Gen*)h; }

int lgo_gen_num_levels(void* h) { return (int)((Gen*)h)->lv.size(); }

// Pointers to level l's new edges (sorted by (src, dst)), deletions and
// weights (null when unweighted); valid until lgo_gen_destroy.
int lgo_gen_level(void* h, int l, const uint32_t** src, const uint32_t** dst, uint64_t* n,
		const uint32_t** dsrc, const uint32_t** ddst, uint64_t* nd, const uint32_t** w) {
	Gen* g = (Gen*)h;
	if (l < 0 || l >= (int)g->lv.size()) return -1;
	const GenLevel& A = g->lv[l];
	*src = A.src.data(); *dst = A.dst.data(); *n = A.src.size();
	*dsrc = A.dsrc.data(); *ddst = A.ddst.data(); *nd = A.dsrc.size();
	*w = A.w.empty() ? nullptr : A.w.data();
	return 0;
}

// Triangle count of the symmetrised, de-duplicated graph given as a
// directed CSR (what lgo_tc counts from a snapshot, and tc_u on the
// flattened store, triangle_counting.h:343-470): the undirected adjacency is
// built, every edge is oriented from the endpoint of lower (degree, id) to
// the higher one, and each triangle u -> v -> w (with u -> w) is found once:
// u's oriented list is marked, then every list of its members is probed.
// *pair_work (may be null) receives the sum over oriented edges (u, v) of
// |N+(u)| + |N+(v)|, the list lengths a merge intersection reads.
int64_t lgo_csr_tc(uint64_t V, const uint64_t* off, const uint32_t* nb, uint64_t* pair_work) {
	std::vector<uint64_t> cnt(V + 1, 0);
	for (uint64_t u = 0; u < V; u++)
		for (uint64_t k = off[u]; k < off[u + 1]; k++)
			if (nb[k] != u) { cnt[u + 1]++; cnt[(uint64_t)nb[k] + 1]++; }
	for (uint64_t v = 0; v < V; v++) cnt[v + 1] += cnt[v];
	std::vector<uint32_t> adj(cnt[V]);
	{
		std::vector<uint64_t> fill(cnt.begin(), cnt.end() - 1);
		for (uint64_t u = 0; u < V; u++)
			for (uint64_t k = off[u]; k < off[u + 1]; k++)
				if (nb[k] != u) { adj[fill[u]++] = nb[k]; adj[fill[nb[k]]++] = (uint32_t)u; }
	}
	std::vector<uint32_t> deg(V);
#pragma omp parallel for schedule(dynamic, 4096)
	for (uint64_t v = 0; v < V; v++) {
		std::sort(adj.begin() + cnt[v], adj.begin() + cnt[v + 1]);
		deg[v] = (uint32_t)(std::unique(adj.begin() + cnt[v], adj.begin() + cnt[v + 1])
				- (adj.begin() + cnt[v]));
	}
	auto before = [&](uint32_t x, uint32_t y) {
		return deg[x] < deg[y] || (deg[x] == deg[y] && x < y);
	};
	// oriented lists, sorted by id
	std::vector<uint64_t> oo(V + 1, 0);
	for (uint64_t v = 0; v < V; v++) {
		uint64_t c = 0;
		for (uint64_t k = cnt[v]; k < cnt[v] + deg[v]; k++) c += before((uint32_t)v, adj[k]);
		oo[v + 1] = oo[v] + c;
	}
	std::vector<uint32_t> on(oo[V]);
#pragma omp parallel for schedule(dynamic, 4096)
	for (uint64_t v = 0; v < V; v++) {
		uint64_t p = oo[v];
		for (uint64_t k = cnt[v]; k < cnt[v] + deg[v]; k++)
			if (before((uint32_t)v, adj[k])) on[p++] = adj[k];
	}
	if (pair_work) {
		uint64_t W = 0;
#pragma omp parallel for schedule(dynamic, 4096) reduction(+:W)
		for (uint64_t u = 0; u < V; u++)
			for (uint64_t k = oo[u]; k < oo[u + 1]; k++)
				W += (oo[u + 1] - oo[u]) + (oo[(uint64_t)on[k] + 1] - oo[on[k]]);
		*pair_work = W;
	}
	// count: mark u's oriented list, then look up each list of its members
	int64_t T = 0;
#pragma omp parallel reduction(+:T)
	{
		std::vector<uint32_t> mark(V, 0);
#pragma omp for schedule(dynamic, 256)
		for (uint64_t u = 0; u < V; u++) {
			const uint32_t stamp = (uint32_t)u + 1;
			for (uint64_t k = oo[u]; k < oo[u + 1]; k++) mark[on[k]] = stamp;
			for (uint64_t k = oo[u]; k < oo[u + 1]; k++) {
				const uint32_t v = on[k];
				for (uint64_t q = oo[v]; q < oo[v + 1]; q++) T += mark[on[q]] == stamp;
			}
		}
	}
	return T;
}

// Personalized PageRank over an in-CSR (lgo_ppr's iteration, all K seeds
// at once and in parallel over vertices): x0 = e_seed, then `iters` times
// x'[t] = (1-d) [t == seed] + d * sum_{w in in(t)} x[w] / outdeg[w], the
// in-neighbours added in the order given, so each column is bit-identical to
// lgo_ppr's.  out is vertex-major, out[v*K + k].
void lgo_csr_ppr(uint64_t V, const uint64_t* in_off, const uint32_t* in_nb,
		const uint32_t* outdeg, const int64_t* seeds, int K, int iters, double d,
		double* out) {
	std::vector<double> x(V * K, 0.0), nx(V * K);
	for (int k = 0; k < K; k++) x[(uint64_t)seeds[k] * K + k] = 1.0;
	for (int it = 0; it < iters; it++) {
#pragma omp parallel
		{
			std::vector<double> S(K);
#pragma omp for schedule(dynamic, 4096)
			for (uint64_t t = 0; t < V; t++) {
				std::fill(S.begin(), S.end(), 0.0);
				for (uint64_t q = in_off[t]; q < in_off[t + 1]; q++) {
					const uint64_t w = in_nb[q];
					for (int k = 0; k < K; k++) S[k] = S[k] + x[w * K + k] / ((double)outdeg[w]);
				}
				for (int k = 0; k < K; k++)
					nx[t * K + k] = ((int64_t)t == seeds[k] ? (1 - d) : 0.0) + d * S[k];
			}
		}
		x.swap(nx);
	}
	std::copy(x.begin(), x.end(), out);
}

// Brandes betweenness centrality over an out-CSR (lgo_bc's restatement of
// bc_random_bfs, bc_random.h:55-111), the sources in parallel: each thread
// runs whole sources with its own level / sigma / delta arrays and its own
// BC sums, which are added at the end (so the order of the per-source adds
// differs from lgo_bc's; FP64, within rounding).
void lgo_csr_bc(uint64_t V, const uint64_t* off, const uint32_t* nb,
		const int64_t* sources, int n, double* bc) {
	std::fill(bc, bc + V, 0.0);
#pragma omp parallel
	{
		std::vector<int32_t> lev(V);
		std::vector<double> sigma(V), delta(V), mine(V, 0.0);
		std::vector<std::vector<uint32_t>> levels;
#pragma omp for schedule(dynamic, 1)
		for (int i = 0; i < n; i++) {
			const int64_t s = sources[i];
			std::fill(lev.begin(), lev.end(), -1);
			std::fill(sigma.begin(), sigma.end(), 0.0);
			levels.assign(1, std::vector<uint32_t>(1, (uint32_t)s));
			lev[s] = 0;
			sigma[s] = 1.0;
			for (int32_t cur = 0; !levels[cur].empty(); cur++) {
				levels.emplace_back();
				for (uint32_t v : levels[cur])
					for (uint64_t q = off[v]; q < off[v + 1]; q++)
						if (lev[nb[q]] < 0) { lev[nb[q]] = cur + 1; levels[cur + 1].push_back(nb[q]); }
				for (uint32_t v : levels[cur])
					for (uint64_t q = off[v]; q < off[v + 1]; q++)
						if (lev[nb[q]] == cur + 1) sigma[nb[q]] += sigma[v];
			}
			for (int32_t cur = (int32_t)levels.size() - 1; cur >= 0; cur--)
				for (uint32_t v : levels[cur]) {
					if ((int64_t)v == s) continue;
					double S = 0.0;
					for (uint64_t q = off[v]; q < off[v + 1]; q++) {
						const uint32_t w = nb[q];
						if (lev[w] == cur + 1) S = S + sigma[v] / sigma[w] * (1 + delta[w]);
					}
					delta[v] = S;
					mine[v] = mine[v] + delta[v];
				}
		}
#pragma omp critical
		for (uint64_t v = 0; v < V; v++) bc[v] += mine[v];
	}
}

} // extern "C"
