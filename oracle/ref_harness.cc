// ref_harness.cc - drives the REFERENCE's own code, compiled from its source
// tree, for the test suite and the CPU baseline.
//
// TEST INFRASTRUCTURE ONLY (see oracle/Makefile).  It includes goatdb/llama's
// headers (-I <reference>/llama/include -I <reference>/benchmark), builds
// levels through the reference's public CSR API - ll_mlcsr_core::init_level,
// init_node, finish_level_vertices, write_value, finish_level_edges and
// update_max_visible_level_lower_only (llama/include/llama/ll_mlcsr_sp.h:
// 624-863, 1375-1627) - and runs the reference benchmark kernels over
// snapshot views ll_mlcsr_ro_graph(master, level)
// (llama/include/llama/ll_mlcsr_graph.h:318-394).
//
// Level sizing: init_level_from_degrees (ll_mlcsr_sp.h:1562-1607) reserves
// continuation space only for vertices with new edges, while init_node also
// writes one for vertices that only lose edges (ll_mlcsr_sp.h:1474-1497),
// which overruns the edge table.  The harness therefore performs the same
// three calls itself (init_level, init_node per vertex,
// finish_level_vertices) and counts every vertex with new or deleted edges.
// No reference source is modified.

#include <llama.h>

#include <time.h>

#include <algorithm>
#include <vector>

#include "benchmarks/bfs.h"
#include "benchmarks/sssp.h"
#include "benchmarks/pagerank.h"
#include "benchmarks/bc_random.h"
#include "benchmarks/triangle_counting.h"
#include "benchmarks/tarjan_scc.h"

// The per-vertex result arrays of the benchmark classes are private members.
// An explicit template instantiation may name a private member (C++ [temp.
// explicit]), which lets the harness read the results without editing the
// reference: Reader<Tag, &Class::member> defines get(Tag) returning the
// member pointer.
template <class Tag, typename Tag::type M>
struct Reader { friend typename Tag::type get(Tag) { return M; } };

struct PrRankTag {
	typedef double* ll_b_pagerank_pull_ext<ll_mlcsr_ro_graph, double>::*type;
	friend type get(PrRankTag);
};
template struct Reader<PrRankTag,
	&ll_b_pagerank_pull_ext<ll_mlcsr_ro_graph, double>::G_pg_rank>;

struct PrPushRankTag {
	typedef double* ll_b_pagerank_push_ext<ll_mlcsr_ro_graph, double>::*type;
	friend type get(PrPushRankTag);
};
template struct Reader<PrPushRankTag,
	&ll_b_pagerank_push_ext<ll_mlcsr_ro_graph, double>::G_pg_rank>;

struct SsspDistTag {
	typedef float* ll_b_sssp_weighted<ll_mlcsr_ro_graph, float>::*type;
	friend type get(SsspDistTag);
};
template struct Reader<SsspDistTag,
	&ll_b_sssp_weighted<ll_mlcsr_ro_graph, float>::G_dist>;

namespace {

struct RefGraph {
	uint64_t V;
	ll_mlcsr_ro_graph* G;
	ll_mlcsr_edge_property<uint32_t>* weight;   // "weight", LL_T_FLOAT, or NULL
};

double now_s() {
	struct timespec ts;
	clock_gettime(CLOCK_MONOTONIC, &ts);
	return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

void build_csr_level(LL_CSR& c, uint64_t V, const std::vector<uint32_t>& cnt_new,
		const std::vector<uint32_t>& cnt_del, int level) {
	size_t max_edges = 0, adj = 0;
	for (uint64_t v = 0; v < V; v++) {
		max_edges += cnt_new[v];
		if (cnt_new[v] > 0 || (level > 0 && cnt_del[v] > 0)) adj++;
	}
	c.init_level(V, adj, max_edges);
	for (uint64_t v = 0; v < V; v++)
		c.init_node(v, cnt_new[v], level == 0 ? 0 : cnt_del[v]);
	c.finish_level_vertices();
}

// Snapshot to run on.  level < 0 (or the latest level) uses the store itself.
// An older level uses the reference's view ll_mlcsr_ro_graph(master, level);
// note that the view copies the master's _maxLevel (ll_mlcsr_sp.h:277), so
// its iterators filter deletions at the master's latest level, not at
// `level`.  The test suite therefore pins snapshot L against a store that
// holds exactly levels 0..L.
struct View {
	ll_mlcsr_ro_graph* clone;
	ll_mlcsr_ro_graph* g;
	View(RefGraph* r, int level) : clone(NULL), g(r->G) {
		if (level >= 0 && level < (int)r->G->num_levels() - 1)
			g = clone = new ll_mlcsr_ro_graph(r->G, level);
	}
	~View() { delete clone; }
};

} // namespace

extern "C" {

void* llref_create(uint64_t V) {
	RefGraph* g = new RefGraph();
	g->V = V;
	g->G = new ll_mlcsr_ro_graph((ll_database*)NULL);
	g->weight = NULL;
	return g;
}

// Append a level with a per-edge weight (uint32, stored as the float edge
// property "weight" that sssp_weighted reads, benchmark.cc:1486-1488).  The
// property level is initialised like a checkpoint does
// (ll_mlcsr_graph.h:1583-1588) and written with cow_write by edge id.
int llref_add_level(void* gp, const uint32_t* src, const uint32_t* dst,
		uint64_t n, const uint32_t* dsrc, const uint32_t* ddst, uint64_t nd);
int llref_add_level_weighted(void* gp, const uint32_t* src, const uint32_t* dst,
		uint64_t n, const uint32_t* dsrc, const uint32_t* ddst, uint64_t nd,
		const uint32_t* w) {
	RefGraph* g = (RefGraph*)gp;
	ll_mlcsr_ro_graph& G = *g->G;
	const int level = (int)G.num_levels();
	if (level == 0)
		g->weight = G.create_uninitialized_edge_property_32("weight", LL_T_FLOAT);
	if (g->weight == NULL) return -3;
	int r = llref_add_level(gp, src, dst, n, dsrc, ddst, nd);
	if (r) return r;
	g->weight->cow_init_level(G.out().max_edges(level));
	// A vertex's new edges are the first fragment its iteration yields and
	// sit at consecutive edge ids in input order, so each vertex needs one
	// find (which returns at once) for its first new edge.
	for (uint64_t i = 0; i < n; ) {
		uint64_t j = i;
		while (j < n && src[j] == src[i]) j++;
		const edge_t e0 = G.out().find(src[i], dst[i]);
		if (e0 == LL_NIL_EDGE || LL_EDGE_LEVEL(e0) != (size_t)level) return -4;
		for (uint64_t k = i; k < j; k++) {
			const edge_t e = e0 + (edge_t)(k - i);
			float f = (float)w[k];
			uint32_t bits;
			memcpy(&bits, &f, 4);
			g->weight->cow_write(e, bits);
		}
		i = j;
	}
	g->weight->cow_finish_level();
	return 0;
}

void llref_destroy(void* gp) {
	RefGraph* g = (RefGraph*)gp;
	delete g->G;
	delete g;
}

int llref_num_levels(void* gp) { return (int)((RefGraph*)gp)->G->num_levels(); }

// Append a level built from new edges (sorted by (src, dst)) and deletions of
// edges live in the latest snapshot.
int llref_add_level(void* gp, const uint32_t* src, const uint32_t* dst,
		uint64_t n, const uint32_t* dsrc, const uint32_t* ddst, uint64_t nd) {
	RefGraph* g = (RefGraph*)gp;
	ll_mlcsr_ro_graph& G = *g->G;
	const uint64_t V = g->V;
	const int level = (int)G.num_levels();
	for (uint64_t i = 1; i < n; i++)
		if (src[i] < src[i - 1] || (src[i] == src[i - 1] && dst[i] <= dst[i - 1]))
			return -1;
	std::vector<int64_t> oe(nd), ie(nd);
	std::vector<uint32_t> onew(V, 0), inew(V, 0), odel(V, 0), idel(V, 0);
	for (uint64_t i = 0; i < nd; i++) {
		if (level == 0) return -1;
		oe[i] = G.out().find(dsrc[i], ddst[i]);
		ie[i] = G.in().find(ddst[i], dsrc[i]);
		if (oe[i] == LL_NIL_EDGE || ie[i] == LL_NIL_EDGE) return -2;
		odel[dsrc[i]]++;
		idel[ddst[i]]++;
	}
	for (uint64_t i = 0; i < n; i++) { onew[src[i]]++; inew[dst[i]]++; }

	// write_value touches only the slots of `node`, so distinct vertices are
	// written in parallel
	std::vector<uint64_t> off(V + 1, 0);
	build_csr_level(G.out(), V, onew, odel, level);
	for (uint64_t v = 0; v < V; v++) off[v + 1] = off[v] + onew[v];
#pragma omp parallel for schedule(dynamic, 4096)
	for (uint64_t v = 0; v < V; v++)
		for (uint64_t k = 0; k < onew[v]; k++)
			G.out().write_value(v, k, (node_t)dst[off[v] + k]);
	G.out().finish_level_edges();

	// in-edges grouped by target, sources ascending (the input is sorted by
	// source, so a stable counting sort by target keeps them ascending)
	build_csr_level(G.in(), V, inew, idel, level);
	{
		for (uint64_t v = 0; v < V; v++) off[v + 1] = off[v] + inew[v];
		std::vector<uint32_t> by_dst(n);
		std::vector<uint64_t> fill(off.begin(), off.end() - 1);
		for (uint64_t i = 0; i < n; i++) by_dst[fill[dst[i]]++] = src[i];
#pragma omp parallel for schedule(dynamic, 4096)
		for (uint64_t v = 0; v < V; v++)
			for (uint64_t k = 0; k < inew[v]; k++)
				G.in().write_value(v, k, (node_t)by_dst[off[v] + k]);
	}
	G.in().finish_level_edges();

	for (uint64_t i = 0; i < nd; i++) {
		G.out().update_max_visible_level_lower_only(oe[i], level);
		G.in().update_max_visible_level_lower_only(ie[i], level);
	}
	return 0;
}

// Copy one level's vertex table (V+1 elements of 16 bytes) and its used edge
// table slots into caller buffers.  With vt == NULL / et == NULL only the
// slot count is returned.
int64_t llref_level_arrays(void* gp, int dir, int level, void* vt, uint64_t* et) {
	RefGraph* g = (RefGraph*)gp;
	LL_CSR& c = dir == 0 ? g->G->out() : g->G->in();
	if (level < 0 || level >= (int)c.num_levels()) return -1;
	uint64_t n_et = c.max_edges(level);
	if (vt) {
		auto* t = c.vertex_table(level);
		for (uint64_t v = 0; v <= g->V; v++) {
			const ll_mlcsr_core__begin_t& e = (*t)[v];
			memcpy((char*)vt + 16 * v, &e, 16);
		}
	}
	if (et) {
		auto* t = c.edge_table(level);
		for (uint64_t i = 0; i < n_et; i++) et[i] = (*t)[i];
	}
	return (int64_t)n_et;
}

// Neighbours of every vertex in snapshot `level`, in the reference's
// iteration order (ll_foreach_out / ll_foreach_in).
uint64_t llref_adjacency(void* gp, int dir, int level, uint64_t* off,
		uint32_t* nbr) {
	RefGraph* g = (RefGraph*)gp;
	View view(g, level);
	ll_mlcsr_ro_graph& S = *view.g;
	uint64_t o = 0;
	for (uint64_t v = 0; v < g->V; v++) {
		off[v] = o;
		ll_edge_iterator it;
		if (dir == 0) {
			S.out_iter_begin(it, v);
			for (edge_t e = S.out_iter_next(it); e != LL_NIL_EDGE; e = S.out_iter_next(it)) {
				if (nbr) nbr[o] = (uint32_t)it.last_node;
				o++;
			}
		} else {
			S.inm_iter_begin(it, v);
			for (node_t w = S.inm_iter_next(it); w != LL_NIL_NODE; w = S.inm_iter_next(it)) {
				if (nbr) nbr[o] = (uint32_t)w;
				o++;
			}
		}
	}
	off[g->V] = o;
	return o;
}

void llref_degrees(void* gp, int level, uint32_t* deg) {
	RefGraph* g = (RefGraph*)gp;
	View view(g, level);
	for (uint64_t v = 0; v < g->V; v++) deg[v] = (uint32_t)view.g->out_degree(v);
}

void llref_set_threads(int n) { if (n > 0) omp_set_num_threads(n); }
int llref_max_threads(void) { return omp_get_max_threads(); }

// "pagerank_double" (benchmark.cc:936-938): returns run() seconds.
double llref_pagerank(void* gp, int level, int iters, double d, double* out) {
	RefGraph* g = (RefGraph*)gp;
	View view(g, level);
	ll_b_pagerank_pull_double<ll_mlcsr_ro_graph> b(iters, d);
	b.initialize(view.g);
	double t0 = now_s();
	b.run();
	double t = now_s() - t0;
	if (out) memcpy(out, b.*get(PrRankTag()), sizeof(double) * g->V);
	b.finalize();
	return t;
}

// "pagerank_double_push" (ll_b_pagerank_push_double, pagerank.h:423-433):
// returns run() seconds.
double llref_pagerank_push(void* gp, int level, int iters, double d, double* out) {
	RefGraph* g = (RefGraph*)gp;
	View view(g, level);
	ll_b_pagerank_push_double<ll_mlcsr_ro_graph> b(iters, d);
	b.initialize(view.g);
	double t0 = now_s();
	b.run();
	double t = now_s() - t0;
	if (out) memcpy(out, b.*get(PrPushRankTag()), sizeof(double) * g->V);
	b.finalize();
	return t;
}

// "sssp_unweighted" levels via u_sssp_bfs (sssp.h:219-300): returns seconds.
double llref_bfs_levels(void* gp, int level, int64_t root, int32_t* dist) {
	RefGraph* g = (RefGraph*)gp;
	View view(g, level);
	ll_mlcsr_ro_graph& S = *view.g;
	for (uint64_t v = 0; v < g->V; v++) dist[v] = INT_MAX - 1;
	node_t r = root;
	dist[r] = 0;
	double t0 = now_s();
	u_sssp_bfs<ll_mlcsr_ro_graph> bfs(S, r, dist);
	bfs.prepare(r);
	bfs.do_bfs_forward();
	return now_s() - t0;
}

// "bfs_count" (bfs.h:117-127): returns the count; *secs = run() seconds.
double llref_bfs_count(void* gp, int level, int64_t root, double* secs) {
	RefGraph* g = (RefGraph*)gp;
	View view(g, level);
	ll_b_bfs<ll_mlcsr_ro_graph> b(root);
	b.initialize(view.g);
	double t0 = now_s();
	double r = b.run();
	if (secs) *secs = now_s() - t0;
	return r;
}

} // extern "C"

extern "C" {

// "sssp_weighted" (ll_b_sssp_weighted<Graph, float>, sssp.h:59-216) from
// `root`; distances written as uint32 (exact: integer weights, sums < 2^24),
// INT_MAX - 1 when unreached.  Returns run() seconds.
double llref_sssp(void* gp, int level, int64_t root, uint32_t* dist) {
	RefGraph* g = (RefGraph*)gp;
	View view(g, level);
	ll_b_sssp_weighted<ll_mlcsr_ro_graph, float> b(root, "weight");
	b.initialize(view.g);
	double t0 = now_s();
	b.run();
	double t = now_s() - t0;
	float* d = b.*get(SsspDistTag());
	for (uint64_t v = 0; v < g->V; v++)
		dist[v] = d[v] < (float)(INT_MAX - 1) ? (uint32_t)d[v] : (uint32_t)(INT_MAX - 1);
	return t;
}

// Brandes BC from explicit sources: the body of ll_b_bc_random::run
// (bc_random.h:158-193) with the given sources in place of
// pick_random_node().  FP32, as in the reference.  Returns seconds.
double llref_bc(void* gp, int level, const int64_t* sources, int n, float* bc) {
	RefGraph* g = (RefGraph*)gp;
	View view(g, level);
	ll_mlcsr_ro_graph& G = *view.g;
	const uint64_t V = g->V;
	float* G_BC = bc;
	std::vector<float> sig(V), del(V);
	float* G_sigma = sig.data();
	float* G_delta = del.data();
	double t0 = now_s();
#pragma omp parallel for
	for (node_t t = 0; t < (node_t)V; t++) G_BC[t] = 0;
	for (int k = 0; k < n; k++) {
		node_t s = sources[k];
#pragma omp parallel for
		for (node_t t = 0; t < (node_t)V; t++) G_sigma[t] = 0;
		G_sigma[s] = 1;
		bc_random_bfs<ll_mlcsr_ro_graph> bfs(G, G_BC, s, G_sigma, G_delta);
		bfs.prepare(s);
		bfs.do_bfs_forward();
		bfs.do_bfs_reverse();
	}
	return now_s() - t0;
}

// "tc_u" (ll_b_triangle_counting_LU, triangle_counting.h:343-470); the store
// must hold exactly one level with symmetric, sorted adjacency.  Returns the
// triangle count; *secs = run() seconds.
int64_t llref_tc_u(void* gp, double* secs) {
	RefGraph* g = (RefGraph*)gp;
	if (g->G->num_levels() != 1) return -1;
	ll_b_triangle_counting_LU<ll_mlcsr_ro_graph> b;
	b.initialize(g->G);
	double t0 = now_s();
	double r = b.run();
	if (secs) *secs = now_s() - t0;
	return (int64_t)r;
}

// "tarjan_scc" (ll_b_tarjan_scc, tarjan_scc.h:121-206), timing only: its
// labels are not true SCCs.  Returns run() seconds.
double llref_tarjan_scc(void* gp, int level) {
	RefGraph* g = (RefGraph*)gp;
	View view(g, level);
	ll_b_tarjan_scc<ll_mlcsr_ro_graph> b;
	b.initialize(view.g);
	double t0 = now_s();
	b.run();
	return now_s() - t0;
}

} // extern "C"
