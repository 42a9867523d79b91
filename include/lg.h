/*
 * lg.h - C ABI of the B200 analytics engine for LLAMA multiversioned CSR stores.
 *
 * The reference (goatdb/llama) exposes its analytics path as header-only C++
 * templates: the read-only multiversion graph `ll_mlcsr_ro_graph`
 * (llama/include/llama/ll_mlcsr_graph.h:83), its iterator vocabulary
 * (llama/include/llama/ll_mlcsr_iterator.h:53-214) and the benchmark task
 * interface `ll_benchmark<Graph>::initialize/run/finalize`
 * (benchmark/benchmarks/benchmark.h:127-319).  This header is the flat,
 * pointer-and-size boundary that replaces those calls on one GPU: the host
 * hands over levels in the reference's own in-memory format (vertex-table
 * elements and 64-bit edge-table slots), and each analytics call runs as
 * hand-written sm_100a kernels over a device-resident mirror of the level
 * stack.
 *
 * Conventions
 *   - Every function returns an lg_status (0 = LG_OK).  On error a message is
 *     kept per thread; read it with lg_last_error().
 *   - Output buffers may be host memory (pageable or pinned) or device memory
 *     of the store's GPU.  With host outputs the call returns after the result
 *     is copied back; with device outputs the work is only enqueued on the
 *     store's stream and lg_store_sync() reports completion and deferred
 *     errors.
 *   - Calls on one store are serialised by the caller (one host thread at a
 *     time, as the reference runs one benchmark at a time); distinct stores
 *     are independent.
 *   - No function falls back to a CPU implementation.  Without a usable GPU
 *     lg_store_create() fails with LG_ECUDA.
 */
#ifndef LG_H_
#define LG_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------------------
 * Status codes.  The reference prints and abort()s (llama/include/llama/
 * ll_utils.h:394-416); the boundary reports instead.
 * ------------------------------------------------------------------------- */
typedef int lg_status;
#define LG_OK        0
#define LG_EINVAL    1   /* bad argument or malformed level                */
#define LG_ENOMEM    2   /* device or pinned host allocation failed        */
#define LG_ECUDA     3   /* CUDA runtime error, or no GPU                  */
#define LG_ETIMEOUT  4   /* an iterative kernel hit its iteration/clock cap */
#define LG_ESTATE    5   /* call not valid in the object's current state   */
#define LG_ENOTSUP   6   /* configuration not supported by this build      */

/* ---------------------------------------------------------------------------
 * Bit layouts shared with the reference (64-bit node ids, LL_DELETIONS on).
 *   edge id   = level << 38 | index          llama/include/llama/ll_mlcsr_helpers.h:55-83
 *   slot      = payload | max_visible_level << 38
 *                                             llama/include/llama/ll_mlcsr_helpers.h:90-114
 *   a slot is visible in snapshot L iff max_visible_level > L
 *   a freshly written slot has max_visible_level = 2^26 - 1
 * ------------------------------------------------------------------------- */
#define LG_BITS_LEVEL        26
#define LG_BITS_INDEX        38
#define LG_NIL_EDGE          ((int64_t)-1)
#define LG_FRESH_MAX_LEVEL   ((1u << LG_BITS_LEVEL) - 1u)
#define LG_EDGE_CREATE(level, index) \
	((int64_t)(((uint64_t)(level) << LG_BITS_INDEX) | (uint64_t)(index)))
#define LG_EDGE_LEVEL(e)     ((uint32_t)((uint64_t)(e) >> LG_BITS_INDEX))
#define LG_EDGE_INDEX(e)     ((uint64_t)(e) & ((1ull << LG_BITS_INDEX) - 1ull))
#define LG_SLOT_PAYLOAD(s)   ((uint64_t)(s) & ((1ull << LG_BITS_INDEX) - 1ull))
#define LG_SLOT_MAX_LEVEL(s) ((uint32_t)((uint64_t)(s) >> LG_BITS_INDEX))

/* Device limits of this build (checked at ingest, LG_ENOTSUP beyond them). */
#define LG_MAX_LEVELS        64          /* levels per store                  */
#define LG_MAX_FRAGMENT_LEN  ((1u << 26) - 1u) /* slots in one level fragment */

/* Unreached vertex in BFS / SSSP outputs: INT_MAX - 1, the value the reference
 * initialises with (benchmark/benchmarks/sssp.h:108, 289-293). */
#define LG_UNREACHED         2147483646

/* Vertex-table element, identical to ll_mlcsr_core__begin_t with
 * LL_PRECOMPUTED_DEGREE (llama/include/llama/ll_mlcsr_helpers.h:141-149):
 * start of this level's adjacency fragment (LG_NIL_EDGE if none), number of
 * slots of that fragment, live out-degree at this level. */
typedef struct lg_vt_entry {
	int64_t  adj_list_start;
	uint32_t level_length;
	uint32_t degree;
} lg_vt_entry;

/* One CSR (out- or in-edges) of one level, as the reference holds it:
 *   vt        max_nodes + 1 elements (the last one is the sentinel written by
 *             finish_level_vertices, llama/include/llama/ll_mlcsr_sp.h:786-808);
 *             alternatively vt_pages, the copy-on-write page table of
 *             ll_mem_array_swcow (512 elements per page,
 *             llama/include/llama/ll_mem_array.h:1019-1032); exactly one of
 *             vt / vt_pages is non-NULL.
 *   slots     the level's edge table, n_slots 64-bit slots (fragments followed
 *             by their 16-byte continuation records for levels > 0,
 *             llama/include/llama/ll_mlcsr_sp.h:1474-1497).
 *   weights   optional per-slot edge property (NULL if none), read by SSSP
 *             like ll_mlcsr_edge_property::get
 *             (llama/include/llama/ll_mlcsr_properties.h:985-1017). */
typedef struct lg_csr_level {
	uint64_t                  max_nodes;
	const lg_vt_entry*        vt;
	const lg_vt_entry* const* vt_pages;
	uint64_t                  n_slots;
	const uint64_t*           slots;
	const uint32_t*           weights;
} lg_csr_level;

/* A deletion recorded in an OLDER level's slot when this level was created:
 * the reference lowers max_visible_level in place
 * (update_max_visible_level_lower_only, llama/include/llama/ll_mlcsr_sp.h:849-863,
 * called from llama/include/llama/ll_writable_graph.h:936-945). */
typedef struct lg_deletion {
	int64_t  edge;               /* LG_EDGE_CREATE(older level, slot index) */
	uint32_t max_visible_level;  /* the new (lowered) value                  */
	uint32_t reserved;
} lg_deletion;

/* Everything one new level adds to the store (the three things a checkpoint
 * changes: a vertex-table level, an edge-table segment, deletion marks in
 * older segments; llama/include/llama/ll_mlcsr_graph.h:1501-1831). */
typedef struct lg_level_desc {
	lg_csr_level        out;
	lg_csr_level        in;           /* in.vt == in.vt_pages == NULL: no in-CSR */
	const lg_deletion*  out_deletions;
	uint64_t            n_out_deletions;
	const lg_deletion*  in_deletions;
	uint64_t            n_in_deletions;
} lg_level_desc;

typedef struct lg_store_opts {
	int   device;        /* CUDA device ordinal                                 */
	void* stream;        /* cudaStream_t to run on, or NULL for a private stream */
	int   reverse_edges; /* 1: levels carry an in-CSR (LL_REVERSE_EDGES)        */
	int   reserved;
} lg_store_opts;

typedef struct lg_store    lg_store;
typedef struct lg_snapshot lg_snapshot;

/* ---------------------------------------------------------------------------
 * Store: device mirror of the level stack.
 * Replaces ll_database / ll_mlcsr_ro_graph ownership of the levels
 * (llama/include/llama/ll_database.h:51-149, ll_mlcsr_graph.h:83).
 * ------------------------------------------------------------------------- */
lg_status lg_store_create(lg_store** store, const lg_store_opts* opts);
lg_status lg_store_destroy(lg_store* store);

/* Append the next level (level number = lg_store_num_levels() before the
 * call).  Mirrors what ll_mlcsr_ro_graph::checkpoint produces
 * (llama/include/llama/ll_mlcsr_graph.h:1501-1831).  Host buffers are copied
 * with pinned staging; the caller may free them on return. */
lg_status lg_store_ingest_level(lg_store* store, const lg_level_desc* level);
int       lg_store_num_levels(const lg_store* store);
lg_status lg_store_max_nodes(const lg_store* store, int level, uint64_t* max_nodes);
lg_status lg_store_sync(lg_store* store);

/* Host output mode of a store (no reference counterpart: the reference's
 * kernels write host arrays in place).
 *   LG_OUTPUT_SYNC  (default) a call with a host output buffer returns after
 *                   the result is in that buffer.
 *   LG_OUTPUT_ASYNC an output of at least LG_ASYNC_MIN_BYTES written to
 *                   page-locked host memory (cudaHostAlloc / cudaHostRegister)
 *                   is staged in a device buffer of the store and copied on a
 *                   second stream of the store, so the copy overlaps the calls
 *                   that follow; the buffer holds the result after
 *                   lg_store_sync().  The caller keeps it alive and does not
 *                   read it before then.  Pageable host memory, smaller
 *                   outputs and the lg_*_result structs are returned as in
 *                   LG_OUTPUT_SYNC.  Two outputs can be in flight; a third
 *                   waits (on the device) for the oldest copy. */
#define LG_OUTPUT_SYNC     0
#define LG_OUTPUT_ASYNC    1
#define LG_ASYNC_MIN_BYTES (1ull << 20)
lg_status lg_store_set_output_mode(lg_store* store, int mode);
/* The stream every call of this store runs on (a cudaStream_t). */
void*     lg_store_stream(const lg_store* store);
/* Device bytes held by the store (levels, deletions, scratch). */
uint64_t  lg_store_device_bytes(const lg_store* store);
/* Number of kernels this store has launched so far (all calls). */
uint64_t  lg_store_launch_count(const lg_store* store);
/* Bytes this store has copied host -> device and device -> host so far
 * (level ingest, deletion lists, results copied to host buffers, and the
 * per-step counters iterative kernels report). */
lg_status lg_store_transfer_bytes(const lg_store* store, uint64_t* h2d,
		uint64_t* d2h);
/* Remove the latest level and the deletion marks it made in older levels,
 * restoring the store to the state before its ingest (the inverse of
 * lg_store_ingest_level; used to age out or re-ingest a snapshot).  Fails with
 * LG_ESTATE while snapshots are open. */
lg_status lg_store_drop_level(lg_store* store);

/* Sliding window (the streaming mode's ll_mlcsr_ro_graph::set_min_level,
 * llama/include/llama/ll_mlcsr_graph.h:560-602 and ll_mlcsr_sp.h:1810-1863,
 * with LL_MIN_LEVEL): levels below min_level age out.  Their device arrays
 * are freed, and every snapshot opened afterwards sees levels min_level..L
 * only: a vertex's fragment chain ends at the first fragment of an older
 * level, as iter_begin / iter_descend end it (ll_mlcsr_sp.h:2021-2026,
 * 2107-2110).  Degrees in such a snapshot are the live edges inside the
 * window.  min_level never decreases and must leave at least the newest level;
 * LG_ESTATE while snapshots are open.  Deleting or re-adding an edge that
 * lives only in aged-out levels sees it as not live. */
lg_status lg_store_set_min_level(lg_store* store, int min_level);
int       lg_store_min_level(const lg_store* store);

/* Build the next level on the device from its edge delta instead of
 * ingesting a level the host built: the vertex tables and edge slots come out
 * as ll_mlcsr_core::init_level_from_degrees / init_node / write_values /
 * finish_level_vertices (llama/include/llama/ll_mlcsr_sp.h:1375-1715) and,
 * for the in-CSR, make_reverse_edges (llama/include/llama/ll_mlcsr_graph.h:
 * 955-1058) lay them out (new edges sorted by (source, target) within a
 * vertex), identical to that level ingested with lg_store_ingest_level; each
 * deleted edge gets its max_visible_level lowered to the new level in the
 * older slot that holds it live (ll_writable_graph.h:936-945).
 *   max_nodes      vertices of the level (>= the previous level's)
 *   src, dst       n_new new edges, any order; no duplicates, none live in
 *                  the previous snapshot
 *   weights        uint32 per new edge, the out-CSR's edge property, or NULL
 *   del_src/dst    n_del edges live in the previous snapshot to delete
 *                  (none at level 0)
 * Arrays may be host or device memory.  On any error the store is unchanged. */
lg_status lg_store_build_level(lg_store* store, uint64_t max_nodes,
		const uint32_t* src, const uint32_t* dst, const uint32_t* weights,
		uint64_t n_new, const uint32_t* del_src, const uint32_t* del_dst,
		uint64_t n_del);

/* Copy level `level` of direction dir (0 out, 1 in) as the device holds it:
 * vt = lg_vt_entry[max_nodes + 1], ids = uint32[n_slots] (the payload of
 * every fragment slot, 0xffffffff elsewhere: continuation records, unused
 * space), weights = uint32[n_slots] (LG_ESTATE if the level has none).  Any
 * output may be NULL; *n_slots (if not NULL) receives the slot count.  No
 * reference counterpart: a readback for checking levels built on the device. */
lg_status lg_store_read_level(lg_store* store, int level, int dir, lg_vt_entry* vt,
		uint32_t* ids, uint32_t* weights, uint64_t* n_slots);

/* ---------------------------------------------------------------------------
 * Snapshots.  A read-only view whose latest level is `level`, with deletions
 * filtered at max_level = level: the snapshot constructor
 * ll_mlcsr_ro_graph(master, level) (llama/include/llama/ll_mlcsr_graph.h:318-394)
 * together with iter_begin(iter, n, level, max_level)
 * (llama/include/llama/ll_mlcsr_sp.h:1994-2053).  Opening resolves every
 * vertex's continuation chain into a fragment list (iter_descend,
 * ll_mlcsr_sp.h:2090-2134) and builds the snapshot's deletion bitset.
 * level = -1 selects the latest level.
 * ------------------------------------------------------------------------- */
lg_status lg_snapshot_open(lg_store* store, int level, lg_snapshot** snap);
/* A snapshot of `level` that sees levels min_level..level only (a sliding
 * window; min_level >= lg_store_min_level).  lg_snapshot_open is this with
 * the store's min level. */
lg_status lg_snapshot_open_window(lg_store* store, int level, int min_level,
		lg_snapshot** snap);
/* Oldest level a snapshot sees. */
lg_status lg_snapshot_min_level(const lg_snapshot* snap, int* min_level);
lg_status lg_snapshot_close(lg_snapshot* snap);
lg_status lg_snapshot_level(const lg_snapshot* snap, int* level);
lg_status lg_snapshot_max_nodes(const lg_snapshot* snap, uint64_t* max_nodes);
/* Number of live edges (sum of out-degrees) of the snapshot. */
lg_status lg_snapshot_num_edges(const lg_snapshot* snap, uint64_t* num_edges);

/* Sizes of one direction (0 out, 1 in) of a snapshot, for byte models. */
typedef struct lg_snapshot_stats {
	uint64_t max_nodes;
	uint64_t live_edges;    /* sum of live degrees                        */
	uint64_t slots;         /* edge-table slots of levels 0..L, continuation
	                           records included                           */
	uint64_t fragment_slots;/* slots covered by the vertices' fragments   */
	uint64_t fragments;     /* (vertex, level) fragments                  */
	uint64_t ranges;        /* 1024-slot work blocks of the slot space    */
	uint64_t deletions;     /* deletion marks visible in the snapshot     */
} lg_snapshot_stats;
lg_status lg_snapshot_get_stats(const lg_snapshot* snap, int dir,
		lg_snapshot_stats* stats);

/* Live out-degree per vertex, uint32[max_nodes]:
 * ll_mlcsr_ro_graph::out_degree (llama/include/llama/ll_mlcsr_graph.h:726-741). */
lg_status lg_out_degrees(lg_snapshot* snap, uint32_t* degrees);
/* Live in-degree per vertex (requires the in-CSR). */
lg_status lg_in_degrees(lg_snapshot* snap, uint32_t* degrees);

/* Materialise the snapshot's adjacency in iteration order: for each vertex,
 * newest fragment first, then older levels, deleted slots skipped - exactly
 * the sequence ll_foreach_out / ll_foreach_in yield
 * (llama/include/llama/ll_mlcsr_iterator.h:186-214).
 * dir = 0 out-edges, 1 in-edges.  offsets: uint64[max_nodes + 1];
 * neighbors: uint32[num edges]; edge_ids: int64 edge ids (may be NULL). */
lg_status lg_snapshot_adjacency(lg_snapshot* snap, int dir, uint64_t* offsets,
		uint32_t* neighbors, int64_t* edge_ids);

/* Flatten one direction (0 out, 1 in) of the snapshot into a single-level
 * CSR kept on the device with the snapshot: the live adjacency in iteration
 * order (the sequence lg_snapshot_adjacency returns), as the task "flatten"
 * builds a one-level graph from all levels on the host
 * (ll_t_flatten, benchmark/tools/flatten.h).  Later traversals of that
 * direction on this snapshot (lg_pagerank_pull; lg_bfs top-down for dir 0,
 * bottom-up for dir 1) read the flat CSR instead of walking fragments and
 * deletion bits; results are unchanged.  Holds about 4 B per live edge (8 B
 * for the out direction of a weighted store, which keeps the weights for
 * SSSP) plus 20 B per vertex of device memory until lg_snapshot_unflatten or
 * lg_snapshot_close, which hand it back to the store: the store keeps up to
 * two released flat CSRs for later flattens (freed by lg_store_destroy).
 * A no-op if the direction is already flat.  LG_ESTATE if dir is 1 and the
 * store keeps no in-CSR. */
lg_status lg_snapshot_flatten(lg_snapshot* snap, int dir);
/* Releases the flat CSRs of both directions (waits for the store's stream). */
lg_status lg_snapshot_unflatten(lg_snapshot* snap);
/* *flat = 1 if direction dir of the snapshot is flattened, else 0. */
lg_status lg_snapshot_is_flat(const lg_snapshot* snap, int dir, int* flat);

/* ---------------------------------------------------------------------------
 * Analytics kernels (the benchmark tasks of benchmark/benchmark.cc:871-946).
 * ------------------------------------------------------------------------- */

/* PageRank, pull direction, FP64: task "pagerank_double",
 * ll_b_pagerank_pull_ext<Graph,double>::run (benchmark/benchmarks/pagerank.h:98-182).
 * pr0 = 1/N with N = max_nodes; each of `iterations` steps sets
 * pr'[t] = (1-d)/N + d * sum_{w in in(t)} pr[w] / out_degree(w); dangling mass
 * is dropped.  ranks: double[max_nodes].  Requires the in-CSR.
 * iterations = 0 returns pr0; the reference's do-while loop
 * (pagerank.h:133-178) runs one iteration when max is 0, so a caller that
 * forwards the reference's -n value passes max(n, 1). */
lg_status lg_pagerank_pull(lg_snapshot* snap, int iterations, double damping,
		double* ranks);

/* PageRank, push direction, FP64: task "pagerank_double_push",
 * ll_b_pagerank_push_ext<Graph,double>::run (benchmark/benchmarks/pagerank.h:258-318).
 * Every vertex t with out-degree > 0 adds pr[t] / out_degree(t) to each
 * out-neighbour's next value (an atomic add, as in the reference), then
 * pr'[t] = (1-d)/N + d * next[t].  Reads only the out-CSR, so it also runs on
 * stores kept without reverse edges.  The summation order follows the atomic
 * schedule: results agree with lg_pagerank_pull within FP64 rounding, not bit
 * for bit.  Uses the flat out-CSR after lg_snapshot_flatten(snap, 0).
 * ranks: double[max_nodes]. */
lg_status lg_pagerank_push(lg_snapshot* snap, int iterations, double damping,
		double* ranks);

/* The same PageRank for callers that cannot let the library allocate device
 * memory (this entry point has no counterpart in the reference).
 * lg_pagerank_pull grows store-owned scratch with cudaMalloc.  Some hosts
 * cannot allow that: a serving process whose device memory is handed out
 * in full to another allocator (a framework's caching allocator or a memory
 * pool sized to the GPU), where a new cudaMalloc fails or forces a
 * device-wide synchronisation, or code that has a rule of no allocation once
 * it has started.  This variant allocates nothing: its per-iteration vectors
 * live in a fixed LG_NOALLOC_SCRATCH_BYTES area compiled into the library,
 * which every GPU that loads the library keeps reserved until the process
 * exits.  The graph must fit: 24 bytes per vertex plus 16 bytes per 1024
 * in-CSR slots <= LG_NOALLOC_SCRATCH_BYTES (about 2.7 million vertices),
 * otherwise LG_EINVAL.  The first call on each device looks up the area's
 * device address (cudaGetSymbolAddress) with that device current; make that
 * first call before any stream capture.  All calls share the one area and
 * leave their values in it; two calls that overlap on the GPU (different
 * streams or stores on the same device) race and must be serialised by the
 * caller.  Same arguments and results as lg_pagerank_pull. */
#define LG_NOALLOC_SCRATCH_BYTES (64ull << 20)
#define LG_NOALLOC_MAX_DEVICES   64
lg_status lg_pagerank_pull_noalloc(lg_snapshot* snap, int iterations,
		double damping, double* ranks);

/* Diagnostic (no reference counterpart): `passes` passes of the PageRank
 * iteration's memory traffic alone over the snapshot's flat in-CSR (lg_snapshot_flatten
 * direction 1 first, else LG_ESTATE): every edge loads its source id and
 * gathers one 8-byte value of a max_nodes vector, in the lane layout of the
 * PageRank kernel, without the row sums.  Timing it gives the speed a kernel
 * that gathers one 8-byte value per edge cannot beat on this snapshot (the
 * floor set by the L1 data path, one wavefront per distinct sector a gather
 * instruction touches); time (2k passes) - (k passes) to leave out the
 * set-up.  *checksum (may be NULL) receives the sum of the values the last
 * pass gathered, to keep the work observable. */
lg_status lg_pagerank_gather_pass(lg_snapshot* snap, int passes, double* checksum);

/* BFS levels from `root`: u_sssp_bfs / ll_b_sssp_unweighted_bfs
 * (benchmark/benchmarks/sssp.h:219-300) over ll_bfs_template
 * (llama/include/llama/ll_bfs_template.h:152-293).  levels: int32[max_nodes],
 * LG_UNREACHED for unreached vertices.  Direction-optimising: switches to
 * bottom-up steps over the in-CSR when the frontier is large (levels are
 * unique, so the result equals the reference's top-down BFS).
 * result (may be NULL): reached = number of reached vertices, the "bfs_count"
 * result (benchmark/benchmarks/bfs.h:117-127); reach_edges = sum of the
 * out-degrees of the reached vertices (the Graph500 edge count used for
 * GTEPS); max_level; and how many steps ran top-down and bottom-up.
 * With the snapshot's in-CSR flat (lg_snapshot_flatten(snap, 1)), or a store
 * without one, the whole traversal is one cooperative launch whose CTAs
 * choose each level's direction on the device and meet at bounded grid
 * barriers (LG_TUNE_BFS_LEVELS; LG_ETIMEOUT if a barrier wait runs out);
 * otherwise a launch sequence per level with the direction chosen on the
 * host.  Both make the same choices and give the same result. */
typedef struct lg_bfs_result {
	uint64_t reached;
	uint64_t reach_edges;
	int32_t  max_level;
	int32_t  top_down_steps;
	int32_t  bottom_up_steps;
	int32_t  reserved;
} lg_bfs_result;

lg_status lg_bfs(lg_snapshot* snap, int64_t root, int32_t* levels,
		lg_bfs_result* result);

/* BFS levels from n_roots roots in one call: the same arrays as n_roots
 * calls of lg_bfs (BFS levels are unique).  The roots share their
 * traversals 64 at a time: every vertex carries one bit per root
 * (bit-parallel multi-source BFS), so an edge visit serves every root whose
 * frontier crosses it at that depth.  levels: int32[n_roots][max_nodes] (row
 * k for roots[k]); results: lg_bfs_result[n_roots] or NULL (top_down_steps /
 * bottom_up_steps count the shared steps of the root's group of 64).  Uses
 * the snapshot's flat CSRs when lg_snapshot_flatten made them.  No reference
 * counterpart as a single call; each row equals task sssp_unweighted. */
lg_status lg_bfs_multi(lg_snapshot* snap, const int64_t* roots, int n_roots,
		int32_t* levels, lg_bfs_result* results);

/* Weighted single-source shortest paths: task "sssp_weighted",
 * ll_b_sssp_weighted::run (benchmark/benchmarks/sssp.h:97-183), whose
 * frontier Bellman-Ford reads G_len[e], the per-slot edge property
 * (llama/include/llama/ll_mlcsr_properties.h:985-1005).  Here the weights are
 * the uint32 per-slot property ingested with the out-CSR (lg_csr_level.weights)
 * and the algorithm is delta-stepping with bucket width `delta`; distances are
 * exact.  dist: uint32[max_nodes], LG_UNREACHED when unreached.  Weights and
 * path lengths must stay below 2^31 - 2.  result (may be NULL): reached
 * vertices (the reference's finalize() value), sum of their out-degrees,
 * largest finite distance, buckets visited, relaxation rounds, relaxations. */
typedef struct lg_sssp_result {
	uint64_t reached;
	uint64_t reach_edges;
	uint32_t max_dist;
	int32_t  buckets;
	int32_t  rounds;
	int32_t  reserved;
	uint64_t relaxations;
} lg_sssp_result;

lg_status lg_sssp_delta(lg_snapshot* snap, int64_t root, uint32_t delta,
		uint32_t* dist, lg_sssp_result* result);

/* Triangle counting on the symmetrised, de-duplicated snapshot: task "tc_u",
 * ll_b_triangle_counting_LU::run (benchmark/benchmarks/triangle_counting.h:
 * 343-470), which needs the graph loaded with -U and flattened to a single
 * sorted level (triangle_counting.h:422-425, benchmark/tools/flatten.h); the
 * flattening happens on the device.  result: the triangle count (each
 * triangle u < v < w once), undirected edges, live arcs read. */
typedef struct lg_tc_result {
	int64_t  triangles;
	uint64_t undirected_edges;
	uint64_t arcs;
} lg_tc_result;

lg_status lg_triangle_count(lg_snapshot* snap, lg_tc_result* result);

/* Strongly connected components: task "tarjan_scc" (ll_b_tarjan_scc,
 * benchmark/benchmarks/tarjan_scc.h:121-206).  The reference's Green-Marl
 * Tarjan uses vertex ids as low-links and does not return true SCCs; this
 * call returns the true partition, each component labelled by its smallest
 * vertex id.  labels: int64[max_nodes].  Requires the in-CSR.  result (may be
 * NULL): number of components, vertices trimmed as singletons up front,
 * colouring rounds and traversal steps. */
typedef struct lg_scc_result {
	uint64_t components;
	uint64_t trimmed;
	int32_t  rounds;
	int32_t  steps;
} lg_scc_result;

lg_status lg_scc(lg_snapshot* snap, int64_t* labels, lg_scc_result* result);

/* Task "avg_teen_cnt" (ll_b_avg_teen_cnt::run,
 * benchmark/benchmarks/avg_teen_cnt.h:96-139): for every vertex n,
 * teen_cnt[n] = number of in-neighbours t with 10 <= age[t] < 20; over the
 * vertices with age[n] > K, average = (float)(sum of teen_cnt / count), 0 if
 * none.  age: int32[max_nodes], the node property "age" of the snapshot
 * (host or device memory); teen_cnt: int32[max_nodes] output, or NULL.  The
 * reference accumulates the sum in int32; teen_sum here is 64-bit (equal
 * while the sum fits 31 bits).  Requires the in-CSR; uses the snapshot's flat
 * in-CSR when lg_snapshot_flatten made one. */
typedef struct lg_teen_result {
	double   average;     /* (float)(teen_sum / vertices), as the task returns it */
	int64_t  teen_sum;    /* sum of teen_cnt over vertices with age > K */
	int64_t  vertices;    /* vertices with age > K */
} lg_teen_result;

lg_status lg_avg_teen_cnt(lg_snapshot* snap, const int32_t* age, int K,
		int32_t* teen_cnt, lg_teen_result* result);

/* Brandes betweenness centrality from explicit sources: the kernel of task
 * "bc_random" (ll_b_bc_random::run, benchmark/benchmarks/bc_random.h:158-193,
 * bc_random_bfs :55-116) with the sources given instead of drawn by
 * pick_random_node(), accumulated in FP64 (the reference uses FP32).
 * Directed, no halving; BC[v] += delta_s[v] for v != s.  bc: double[max_nodes].
 * lg_bc runs one source after another; lg_bc_batched runs 64 sources per
 * pass (one edge traversal serves 64 BFSs) and returns the same values up to
 * FP64 summation order. */
lg_status lg_bc(lg_snapshot* snap, const int64_t* sources, int n_sources,
		double* bc);
lg_status lg_bc_batched(lg_snapshot* snap, const int64_t* sources, int n_sources,
		double* bc);

/* Personalized PageRank for K single-vertex seeds, evaluated on n_snaps
 * snapshots of one store in a single CUDA-graph launch.  The reference has no
 * personalized variant: this is the pull iteration of pagerank_double
 * (benchmark/benchmarks/pagerank.h:120-169) with the uniform teleport
 * (1-d)/N replaced, per column k, by (1-d) on seed k; x0 = e_seed, fixed
 * iteration count, dangling mass dropped.  K is a multiple of 32, <= 256.
 * out: double[n_snaps][max_nodes][K] (row-major, column k = seed k). */
lg_status lg_ppr(lg_snapshot* const* snaps, int n_snaps, const int64_t* seeds,
		int K, int iterations, double damping, double* out);

/* Differentiable weighted PageRank (no reference counterpart; the pull
 * iteration of pagerank.h:120-169 with per-edge weights and a teleport
 * vector).  Forward: x = (1-d) teleport + d P^T x from x = teleport until
 * sum |x' - x| < tol (or max_iter), P(w->t) = weights[p] where p is the
 * edge's position in the snapshot's out-adjacency order (lg_snapshot_adjacency
 * dir 0); the caller normalises rows if it wants a stochastic P.  x:
 * double[max_nodes].  If tape is non-NULL the converged x is kept for
 * lg_pagerank_bwd, which solves the transposed fixed point
 * lambda = dL/dx + d P lambda (implicit differentiation, no stored iterates)
 * and returns dL/dweights (double[num_edges], same order) = d lambda[t] x[w]
 * and dL/dteleport (double[max_nodes]) = (1-d) lambda; either may be NULL.
 * Free the tape with lg_adjoint_free before closing the snapshot. */
typedef struct lg_adjoint lg_adjoint;
typedef struct lg_fixed_point_result {
	int32_t iterations;
	int32_t reserved;
	double  residual;   /* sum |x' - x| of the last iteration */
} lg_fixed_point_result;

lg_status lg_pagerank_fwd(lg_snapshot* snap, const double* weights,
		const double* teleport, double damping, double tol, int max_iter,
		double* x, lg_adjoint** tape, lg_fixed_point_result* result);
lg_status lg_pagerank_bwd(lg_adjoint* tape, const double* dldx, double* dldw,
		double* dldteleport, lg_fixed_point_result* result);
lg_status lg_adjoint_free(lg_adjoint* tape);

/* ---------------------------------------------------------------------------
 * Launch parameters (no counterpart in the reference, whose OpenMP kernels
 * have no launch shapes).  Each GPU has a table of values that the kernels
 * read when they are launched; lg_tune_set pins one, lg_autotune measures
 * candidates on a snapshot and keeps the fastest.  Out-of-range values are
 * rejected with LG_EINVAL; every value gives the same results, only the
 * speed changes.
 * ------------------------------------------------------------------------- */
/* Flat-CSR sweeps (PageRank pull, the adjoint's solves): resident CTAs (of
 * 8 warps) per SM of a persistent sweep, each warp looping over 256-edge
 * tiles; 0 = one CTA per 4 tiles, each warp one tile. */
#define LG_TUNE_PR_CTAS_PER_SM  0
/* Personalized PageRank: columns per pass (a multiple of 32; the K columns
 * run in passes of this many, each pass all iterations), default 256. */
#define LG_TUNE_PPR_KTILE       1
/* Personalized PageRank: in-CSR slots per warp range, default 2048. */
#define LG_TUNE_PPR_RANGE       2
/* Delta-stepping SSSP: queue slots per warp range, default 1024. */
#define LG_TUNE_SSSP_RANGE      3
/* Multi-source BFS and batched BC bottom-up steps: in-degree above which a
 * warp, not a thread, scans a vertex's in-edges, default 512. */
#define LG_TUNE_MS_HEAVY        4
/* PageRank's tile kernel (LG_TUNE_PR_CTAS_PER_SM = 0): 8 = the build whose
 * registers are capped for 64 resident warps per SM; any other
 * value = the build the compiler sizes freely (default 0). */
#define LG_TUNE_PR_TILE_OCC     5
/* Delta-stepping SSSP: 1 = the rounds of a bucket relax only the light edges
 * (weight < delta) of the near queue and the vertices settled in the bucket
 * relax their heavy edges once when it drains, over a copy of the snapshot's
 * out-CSR split per row (built on the first call for a delta, 8 bytes per
 * live edge, kept with the snapshot); 0 = every round relaxes every edge of
 * the near queue.  Default 0 (measured faster on the R-MAT workloads). */
#define LG_TUNE_SSSP_SPLIT      6
/* One-root BFS (lg_bfs) with the snapshot's in-CSR flat (or no in-CSR):
 * 1 = every level in one cooperative launch whose CTAs choose the direction
 * on the device and meet at grid barriers; 0 = a launch sequence per level
 * with the direction chosen on the host.  Default 1. */
#define LG_TUNE_BFS_LEVELS      7
/* Delta-stepping SSSP: 1 = all rounds, bucket splits and heavy phases in one
 * cooperative launch whose CTAs apply the host loop's rules on the device
 * and meet at bounded grid barriers; 0 = a launch sequence per step with the
 * host reading the counters back.  Default 0: on the R-MAT workloads the one
 * launch gains 3-8 % with LG_TUNE_SSSP_SPLIT and loses 8 % without (its
 * relaxation loop holds fewer warps per SM than the per-step kernel). */
#define LG_TUNE_SSSP_LEVELS     8
#define LG_TUNE_COUNT           9
#define LG_TUNE_MAX_DEVICES     64
lg_status lg_tune_get(int device, int key, int64_t* value);
lg_status lg_tune_set(int device, int key, int64_t value);
lg_status lg_tune_reset(int device);

/* The autotuner: for every tunable whose bit (1u << key) is set in `keys`,
 * sets each candidate value on the snapshot's GPU in turn, times the call
 * that reads it on this snapshot (a warm-up call, then the median of three
 * timed with CUDA events; PageRank pull, PPR with 256 seeds, SSSP,
 * multi-source BFS and four one-root BFS from vertices of the snapshot), and
 * keeps the fastest.
 * Tunables that the snapshot cannot exercise (SSSP without weights, the
 * others without an in-CSR) are skipped, and so are the PPR ones when three
 * max_nodes x 256 FP64 blocks do not fit in half of the free device memory.  trials (may be NULL)
 * receives one entry per candidate measured, up to max_trials; n_trials the
 * count.  Allocates its own probe buffers; the snapshot is not changed.  The
 * PageRank and BFS probes run over the flat in-CSR: when the snapshot has
 * none, one is made for them (lg_snapshot_flatten's memory) and released
 * when the probes end; where it does not fit, the PageRank probes flatten
 * per call and LG_TUNE_MS_HEAVY and LG_TUNE_BFS_LEVELS, read only with a
 * flat in-CSR, are skipped. */
typedef struct lg_tune_trial {
	int32_t key;
	int32_t chosen;    /* 1 for the value kept */
	int64_t value;
	double  ms;        /* median time of the probe call */
} lg_tune_trial;
lg_status lg_autotune(lg_snapshot* snap, unsigned keys, lg_tune_trial* trials,
		int max_trials, int* n_trials);

/* ---------------------------------------------------------------------------
 * Errors.
 * ------------------------------------------------------------------------- */
/* Copies the calling thread's last error message (NUL-terminated, truncated
 * to len); returns the message length. */
size_t    lg_last_error(char* buf, size_t len);
const char* lg_status_string(lg_status status);
/* Version of this library, "major.minor.patch". */
const char* lg_version(void);

#ifdef __cplusplus
}
#endif

#endif /* LG_H_ */
