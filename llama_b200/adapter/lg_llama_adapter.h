// lg_llama_adapter.h - the LLAMA-side binding of the B200 engine: what a
// goatdb/llama build adds to call liblg.  Header-only C++ over LLAMA's own
// types, included after <llama.h> and benchmark/benchmarks/benchmark.h.
//
// 1. lg_llama_ingest_level hands level l of a read-only graph to a device
//    store exactly as ll_mlcsr_core holds it: each direction's vertex-table
//    level (ll_mlcsr_core__begin_t, llama/include/llama/ll_mlcsr_helpers.h:
//    141-149, read through the ll_mem_array_swcow table,
//    ll_mem_array.h:1019-1032) and its edge table (ll_et_array,
//    ll_edge_table.h:54-208), plus the deletion marks made in levels that
//    are already on the device.
// 2. ll_b_pagerank_pull_gpu is a task of the benchmark interface
//    (ll_benchmark<Graph>, benchmark/benchmarks/benchmark.h:127-319) that
//    runs "pagerank_double" (pagerank.h:98-182) on the device: same
//    constructor arguments, same per-vertex result array and the same
//    finalize() value (the sum of the ranks), so it registers beside the CPU
//    row of g_runnable_things (benchmark/benchmark.cc:871-968).
#ifndef LG_LLAMA_ADAPTER_H_
#define LG_LLAMA_ADAPTER_H_

#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#include <vector>

#include "lg.h"

// One CSR direction of level l, its vertex table copied out of the COW table.
template <class CSR>
inline lg_csr_level lg_llama_csr_level(CSR& c, int l, size_t V, std::vector<lg_vt_entry>& vt) {
	vt.resize(V + 1);
	auto& t = *c.vertex_table(l);
	for (size_t v = 0; v <= V; v++) {
		const auto& e = t[v];
		vt[v].adj_list_start = e.adj_list_start;
		vt[v].level_length = (uint32_t)e.level_length;
		vt[v].degree = (uint32_t)e.degree;
	}
	lg_csr_level d;
	d.max_nodes = V;
	d.vt = vt.data();
	d.vt_pages = NULL;
	d.n_slots = c.max_edges(l);
	d.slots = d.n_slots ? (const uint64_t*)&(*c.edge_table(l))[0] : NULL;
	d.weights = NULL;
	return d;
}

// Ingest level l of G into `store`.  out_marks / in_marks: the deletions
// this level made in levels already ingested (the (edge, level) pairs given
// to update_max_visible_level_lower_only, ll_writable_graph.h:936-945);
// marks already present in the slots of levels ingested after them are read
// from the slots, so a store filled once a graph is complete needs none.
// Aborts on error, LLAMA's convention (ll_utils.h:394-416).
template <class Graph>
inline void lg_llama_ingest_level(lg_store* store, Graph& G, int l,
		const std::vector<lg_deletion>& out_marks = std::vector<lg_deletion>(),
		const std::vector<lg_deletion>& in_marks = std::vector<lg_deletion>()) {
	const size_t V = G.max_nodes();
	std::vector<lg_vt_entry> vo, vi;
	lg_level_desc d;
	d.out = lg_llama_csr_level(G.out(), l, V, vo);
	d.in = lg_llama_csr_level(G.in(), l, V, vi);
	d.out_deletions = out_marks.empty() ? NULL : out_marks.data();
	d.n_out_deletions = out_marks.size();
	d.in_deletions = in_marks.empty() ? NULL : in_marks.data();
	d.n_in_deletions = in_marks.size();
	if (lg_store_ingest_level(store, &d) != LG_OK) {
		char msg[256];
		lg_last_error(msg, sizeof msg);
		fprintf(stderr, "GPU ingest of level %d failed: %s\n", l, msg);
		abort();
	}
}

// Task "pagerank_double" on the device: run() opens the latest snapshot of
// the store, runs lg_pagerank_pull into the task's own rank array and
// returns 0 (NaN if the call failed); finalize() returns the sum of the
// ranks, like ll_b_pagerank_pull_ext::finalize (pagerank.h:190-199).
template <class Graph>
class ll_b_pagerank_pull_gpu : public ll_benchmark<Graph> {
	int32_t max;
	double d;
	double* G_pg_rank;
	lg_store* store;

public:
	ll_b_pagerank_pull_gpu(lg_store* s, int32_t m, double damping = 0.85)
		: ll_benchmark<Graph>("PageRank<double> - Pull (B200)"), max(m), d(damping),
		  G_pg_rank(NULL), store(s) {
		this->create_auto_array_for_nodes(G_pg_rank);
	}

	virtual double run(void) {
		lg_snapshot* snap = NULL;
		if (lg_snapshot_open(store, -1, &snap) != LG_OK) return NAN;
		// the reference's do-while loop runs one iteration when max is 0
		lg_status st = lg_pagerank_pull(snap, max > 0 ? max : 1, d, G_pg_rank);
		lg_snapshot_close(snap);
		return st == LG_OK ? 0 : NAN;
	}

	virtual double finalize(void) {
		double s = 0;
		for (node_t n = 0; n < this->_graph->max_nodes(); n++) s += G_pg_rank[n];
		return s;
	}

	virtual void print_results(FILE* f) {
		print_results_part(f, this->_graph, G_pg_rank);
	}

	const double* ranks() const { return G_pg_rank; }
};

#endif // LG_LLAMA_ADAPTER_H_
