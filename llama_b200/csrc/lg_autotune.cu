// lg_autotune.cu - picks launch parameters (lg_tune.cpp) by measuring them.
//
// For every requested tunable, each candidate value is set on the snapshot's
// GPU and the call that reads it is run on the snapshot: one warm-up call,
// then the median of three calls timed with CUDA events on the store's
// stream.  The fastest value stays set.  Tunables are taken one after the
// other, each measured with the values already chosen for the others.  The
// probes write into device buffers of their own, so the snapshot and the
// caller's data are untouched; every value computes the same results.
#include "lg_device.cuh"
#include "lg_flat.cuh"
#include "lg_tune.h"

#include <algorithm>
#include <functional>
#include <vector>

using namespace lg;

namespace {

struct Probe {
	int key;
	std::vector<int64_t> values;
	std::function<lg_status()> call;
};

lg_status time_call(lg_store* s, const std::function<lg_status()>& call, double* ms) {
	cudaStream_t st = s->stream;
	cudaEvent_t e0 = nullptr, e1 = nullptr;
	LG_CUDA(cudaEventCreate(&e0), "event");
	cudaError_t ce = cudaEventCreate(&e1);
	if (ce != cudaSuccess) { cudaEventDestroy(e0); return cuda_status(ce, "event"); }
	lg_status r = call();                       // warm-up
	std::vector<float> t;
	for (int i = 0; i < 3 && !r; i++) {
		ce = cudaEventRecord(e0, st);
		if (ce == cudaSuccess) { r = call(); ce = cudaEventRecord(e1, st); }
		if (ce == cudaSuccess) ce = cudaEventSynchronize(e1);
		float x = 0;
		if (ce == cudaSuccess) ce = cudaEventElapsedTime(&x, e0, e1);
		if (ce != cudaSuccess && !r) r = cuda_status(ce, "autotune timing");
		t.push_back(x);
	}
	cudaEventDestroy(e0);
	cudaEventDestroy(e1);
	if (r) return r;
	std::sort(t.begin(), t.end());
	*ms = t[t.size() / 2];
	return LG_OK;
}

} // namespace

extern "C" lg_status lg_autotune(lg_snapshot* sn, unsigned keys, lg_tune_trial* trials,
		int max_trials, int* n_trials) {
	clear_error();
	if (!sn) return set_error(LG_EINVAL, "null snapshot");
	if (n_trials) *n_trials = 0;
	lg_store* s = sn->store;
	LG_CUDA(cudaSetDevice(s->device), "cudaSetDevice");
	const uint64_t V = sn->V;
	// probe inputs: 64 (or 256) vertices with out-edges, evenly spaced
	std::vector<uint32_t> deg(V);
	LG_TRY(lg_out_degrees(sn, deg.data()));
	std::vector<int64_t> has;
	for (uint64_t v = 0; v < V; v++) if (deg[v]) has.push_back((int64_t)v);
	if (has.empty()) return set_error(LG_EINVAL, "the snapshot has no edges");
	auto pick = [&](size_t n) {
		std::vector<int64_t> r;
		for (size_t i = 0; i < n; i++) r.push_back(has[(i * has.size()) / n]);
		return r;
	};
	const std::vector<int64_t> roots = pick(64), seeds = pick(256);
	bool weighted = true;
	for (int l = sn->min_level; l <= sn->level; l++)
		if (s->out.levels[l]->n_fragment_slots > 0 && !s->out.levels[l]->w.p) weighted = false;

	// PPR probes hold three V x 256 FP64 blocks: only where they fit in half
	// of the free device memory
	size_t free_b = 0, total_b = 0;
	LG_CUDA(cudaMemGetInfo(&free_b, &total_b), "cudaMemGetInfo");
	const uint64_t ppr_block = V * 256ull * sizeof(double);
	const bool ppr_fits = 3 * ppr_block <= free_b / 2;
	const bool want_ppr = (keys & ((1u << LG_TUNE_PPR_KTILE) | (1u << LG_TUNE_PPR_RANGE)))
			&& ppr_fits && sn->in.present;
	DevBuf out;
	LG_TRY(out.reserve(std::max<uint64_t>(want_ppr ? ppr_block : V * sizeof(double),
			V * 64 * sizeof(int32_t))));
	double* dout = out.as<double>();
	int32_t* iout = out.as<int32_t>();
	lg_snapshot* one[1] = {sn};
	// PageRank's sweeps, the multi-source bottom-up steps that read
	// LG_TUNE_MS_HEAVY and the one-launch BFS run over the flat in-CSR: a
	// snapshot without one gets
	// one for the probes (so a PageRank probe times the sweeps, not a flatten
	// per call) and gives it back when they end.  Without the memory for it
	// the PageRank probes build their own per call and the MS_HEAVY and
	// BFS_LEVELS probes, whose values only the flat kernels read, are skipped.
	const unsigned in_keys = (1u << LG_TUNE_PR_CTAS_PER_SM) | (1u << LG_TUNE_PR_TILE_OCC) |
			(1u << LG_TUNE_MS_HEAVY) | (1u << LG_TUNE_BFS_LEVELS);
	struct FlatGuard {
		lg_snapshot* sn = nullptr;
		~FlatGuard() {
			if (!sn) return;
			cudaStreamSynchronize(sn->store->stream);
			lg_flat_release(sn->store, sn->flat[1]);
			sn->flat[1] = nullptr;
		}
	} made_in;
	if ((keys & in_keys) && sn->in.present && !sn->flat[1]) {
		if (lg_snapshot_flatten(sn, 1) == LG_OK) made_in.sn = sn;
		else clear_error();
	}
	std::vector<Probe> probes;
	if ((keys & (1u << LG_TUNE_PR_CTAS_PER_SM)) && sn->in.present)
		probes.push_back({LG_TUNE_PR_CTAS_PER_SM, {0, 4, 5, 6},
			[=]() { return lg_pagerank_pull(sn, 6, 0.85, dout); }});
	if ((keys & (1u << LG_TUNE_PR_TILE_OCC)) && sn->in.present)
		probes.push_back({LG_TUNE_PR_TILE_OCC, {0, 8},
			[=]() { return lg_pagerank_pull(sn, 6, 0.85, dout); }});
	if ((keys & (1u << LG_TUNE_PPR_KTILE)) && want_ppr)
		probes.push_back({LG_TUNE_PPR_KTILE, {32, 64, 128, 256},
			[=, &seeds]() { return lg_ppr(one, 1, seeds.data(), 256, 4, 0.85, dout); }});
	if ((keys & (1u << LG_TUNE_PPR_RANGE)) && want_ppr)
		probes.push_back({LG_TUNE_PPR_RANGE, {1024, 2048, 4096},
			[=, &seeds]() { return lg_ppr(one, 1, seeds.data(), 256, 4, 0.85, dout); }});
	if ((keys & (1u << LG_TUNE_SSSP_RANGE)) && weighted)
		probes.push_back({LG_TUNE_SSSP_RANGE, {512, 1024, 2048, 4096},
			[=, &roots]() {
				return lg_sssp_delta(sn, roots[0], 32, (uint32_t*)iout, nullptr);
			}});
	if ((keys & (1u << LG_TUNE_SSSP_SPLIT)) && weighted)
		probes.push_back({LG_TUNE_SSSP_SPLIT, {0, 1},
			[=, &roots]() {
				return lg_sssp_delta(sn, roots[0], 32, (uint32_t*)iout, nullptr);
			}});
	if ((keys & (1u << LG_TUNE_SSSP_LEVELS)) && weighted)
		probes.push_back({LG_TUNE_SSSP_LEVELS, {0, 1},
			[=, &roots]() {
				return lg_sssp_delta(sn, roots[0], 32, (uint32_t*)iout, nullptr);
			}});
	if ((keys & (1u << LG_TUNE_MS_HEAVY)) && sn->flat[1])
		probes.push_back({LG_TUNE_MS_HEAVY, {128, 256, 512, 1024, 4096},
			[=, &roots]() {
				return lg_bfs_multi(sn, roots.data(), (int)roots.size(), iout, nullptr);
			}});
	if ((keys & (1u << LG_TUNE_BFS_LEVELS)) && (sn->flat[1] || !sn->in.present))
		probes.push_back({LG_TUNE_BFS_LEVELS, {0, 1},
			[=, &roots]() {
				lg_status r = LG_OK;
				for (int i = 0; i < 4 && !r; i++) r = lg_bfs(sn, roots[i * 16], iout, nullptr);
				return r;
			}});
	int nt = 0;
	for (const Probe& p : probes) {
		int64_t best_v = 0;
		double best = -1;
		const int first = nt;
		for (int64_t v : p.values) {
			LG_TRY(lg_tune_set(s->device, p.key, v));
			double ms = -1;
			lg_status r = time_call(s, p.call, &ms);
			if (r) return r;
			if (best < 0 || ms < best) { best = ms; best_v = v; }
			if (trials && nt < max_trials) {
				trials[nt].key = p.key;
				trials[nt].chosen = 0;
				trials[nt].value = v;
				trials[nt].ms = ms;
			}
			nt++;
		}
		LG_TRY(lg_tune_set(s->device, p.key, best_v));
		for (int i = first; i < nt && trials && i < max_trials; i++)
			trials[i].chosen = trials[i].value == best_v;
	}
	if (n_trials) *n_trials = std::min(nt, trials ? max_trials : nt);
	return LG_OK;
}
