// adapter_harness.cc - compiles the LLAMA-side binding of the engine
// (llama_b200/adapter/lg_llama_adapter.h) against the reference's own
// headers and runs it on a reference store, beside the reference's CPU task.
//
// TEST INFRASTRUCTURE ONLY (see oracle/Makefile): one translation unit with
// ref_harness.cc, so the store is built by the same code the oracle checks
// use, linked with llama_b200/liblg.so.  The tests call llref_gpu_pagerank,
// which is what a LLAMA maintainer's `benchmark -r pagerank_double_gpu` row
// would run: fill a device store from the graph's levels
// (lg_llama_ingest_level), then initialize / run / finalize the
// ll_b_pagerank_pull_gpu task; the reference's ll_b_pagerank_pull_double task
// (benchmark/benchmarks/pagerank.h:98-216) runs on the same graph for the
// comparison.
#include "ref_harness.cc"

#include "lg_llama_adapter.h"

extern "C" {

// out[0] = GPU task run(), out[1] = its finalize(), out[2] = the CPU task's
// finalize(); ranks_gpu / ranks_cpu (may be NULL) receive the per-vertex
// ranks.  Returns 0, or -1 when no device store can be created.
int llref_gpu_pagerank(void* gp, int iters, double d, double* ranks_gpu,
		double* ranks_cpu, double* out) {
	RefGraph* g = (RefGraph*)gp;
	ll_mlcsr_ro_graph& G = *g->G;
	lg_store_opts opts;
	opts.device = 0;
	opts.stream = NULL;
	opts.reverse_edges = 1;
	opts.reserved = 0;
	lg_store* store = NULL;
	if (lg_store_create(&store, &opts) != LG_OK) return -1;
	for (int l = 0; l < (int)G.num_levels(); l++) lg_llama_ingest_level(store, G, l);

	ll_b_pagerank_pull_gpu<ll_mlcsr_ro_graph> gpu(store, iters, d);
	gpu.initialize(&G);
	out[0] = gpu.run();
	out[1] = gpu.finalize();
	if (ranks_gpu) memcpy(ranks_gpu, gpu.ranks(), sizeof(double) * g->V);

	ll_b_pagerank_pull_double<ll_mlcsr_ro_graph> cpu(iters, d);
	cpu.initialize(&G);
	cpu.run();
	out[2] = cpu.finalize();
	if (ranks_cpu) memcpy(ranks_cpu, cpu.*get(PrRankTag()), sizeof(double) * g->V);
	lg_store_destroy(store);
	return 0;
}

} // extern "C"
