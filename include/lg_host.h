/*
 * lg_host.h - host-side producer of LLAMA levels for the lg_* device engine.
 *
 * The reference builds read-only levels on the host with
 * ll_mlcsr_core::init_level_from_degrees / init_node / write_value
 * (llama/include/llama/ll_mlcsr_sp.h:1375-1715) and marks deletions in older
 * slots with update_max_visible_level_lower_only (ll_mlcsr_sp.h:849-863).
 * lg_hgraph does the same construction, in parallel, and keeps every level in
 * the reference's byte layout so that lg_store_ingest_level() receives
 * exactly what a LLAMA ll_mlcsr_ro_graph holds.  The seeded generators below
 * stand in for the reference's loaders (llama/include/llama/loaders/) with
 * the synthetic R-MAT / Kronecker inputs the benchmarks are quoted on.
 */
#ifndef LG_HOST_H_
#define LG_HOST_H_

#include "lg.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct lg_hgraph lg_hgraph;

/* Multiversion host graph with max_nodes vertices (out-CSR, plus in-CSR when
 * reverse_edges != 0, like LL_REVERSE_EDGES). */
lg_status lg_hgraph_create(lg_hgraph** g, uint64_t max_nodes, int reverse_edges);
lg_status lg_hgraph_destroy(lg_hgraph* g);

/* Append one level (a checkpoint).  new edges: src/dst pairs that are not
 * live in the latest snapshot (any order; each fragment is written sorted by
 * target, as the reference loaders do, llama/include/llama/loaders/
 * ll_load_utils.h:649-784).  deletions: pairs live in the latest snapshot;
 * their slots get max_visible_level = the new level number.  weights: one
 * uint32 per new edge (NULL = none), stored as a per-slot edge property. */
lg_status lg_hgraph_add_level(lg_hgraph* g,
		const uint32_t* src, const uint32_t* dst, uint64_t n_new,
		const uint32_t* del_src, const uint32_t* del_dst, uint64_t n_del,
		const uint32_t* weights);
int       lg_hgraph_num_levels(const lg_hgraph* g);
uint64_t  lg_hgraph_max_nodes(const lg_hgraph* g);

/* Descriptor of one level in the reference layout; the pointers stay valid
 * until the graph is destroyed.  The deletion lists are the marks this level
 * made in older levels. */
lg_status lg_hgraph_level_desc(lg_hgraph* g, int level, lg_level_desc* desc);

/* Ingest levels [first, num_levels) into a device store (which must already
 * hold levels [0, first)). */
lg_status lg_hgraph_ingest(lg_hgraph* g, lg_store* store, int first);

/* The inputs a level was built from (sorted by src then dst), for feeding the
 * same level to another implementation.  Pointers stay valid until destroy. */
lg_status lg_hgraph_level_input(lg_hgraph* g, int level,
		const uint32_t** src, const uint32_t** dst, uint64_t* n_new,
		const uint32_t** del_src, const uint32_t** del_dst, uint64_t* n_del,
		const uint32_t** weights);

/* ---------------------------------------------------------------------------
 * Seeded synthetic inputs.
 * ------------------------------------------------------------------------- */
#define LG_GEN_RMAT       0   /* R-MAT, no noise, ids as generated          */
#define LG_GEN_KRONECKER  1   /* Graph500-style: R-MAT quadrant recursion,
                                 vertex ids scrambled by a seeded bijection */

typedef struct lg_graph_spec {
	int      kind;             /* LG_GEN_RMAT or LG_GEN_KRONECKER             */
	int      scale;            /* 2^scale vertices                            */
	double   edge_factor;      /* edge_factor * 2^scale draws                 */
	double   a, b, c;          /* quadrant probabilities, d = 1 - a - b - c   */
	uint64_t seed;
	int      symmetrize;       /* store both arcs of every edge               */
	int      num_levels;       /* >= 1                                        */
	double   level0_fraction;  /* share of edges in level 0; the rest is split
	                              evenly over levels 1 .. num_levels-1        */
	double   delete_fraction;  /* share of live edges deleted at each level>0 */
	uint64_t split_seed;
	uint32_t weight_max;       /* 0: no weights; else uint32 in [1, weight_max] */
	uint64_t weight_seed;
} lg_graph_spec;

/* Draw edge_factor * 2^scale edges, drop self-loops and duplicates (and, with
 * symmetrize, add the reverse arcs).  Writes the unique edges sorted by
 * (src, dst) into src/dst (capacity entries each; capacity must be at least
 * the number of draws, times 2 with symmetrize) and their count to n. */
lg_status lg_gen_edges(const lg_graph_spec* spec, uint32_t* src, uint32_t* dst,
		uint64_t capacity, uint64_t* n);

/* Generate the edges of `spec`, split them into spec->num_levels levels with
 * the deletions the spec asks for, and append those levels to g (which must
 * be empty and have 2^scale vertices). */
lg_status lg_hgraph_build(lg_hgraph* g, const lg_graph_spec* spec);

/* The weight the generator assigns to edge (src, dst) under a spec. */
uint32_t  lg_gen_weight(const lg_graph_spec* spec, uint32_t src, uint32_t dst);

#ifdef __cplusplus
}
#endif

#endif /* LG_HOST_H_ */
