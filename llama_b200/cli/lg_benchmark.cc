// lg_benchmark - drop-in for LLAMA's `benchmark -r <task> FILE...`
// (benchmark/benchmark.cc:976-2031) running the tasks on a B200 through the
// C ABI.
//
// As in the reference, every input file becomes one level (checkpoint) of
// the multiversion store (benchmark.cc:1614-1663).  A file is an edge list:
// "src dst [weight]" per line, '#' or '%' starts a comment; a line
// "- src dst" deletes an edge live in the previous levels (this is how a
// level records deletions; the reference gets them from ll_writable_graph).
// The task runs on the latest loaded snapshot and the program prints
// "Return value: %lf" with the value the reference task's finalize() /
// run() returns (benchmark.cc:1140-1154, 2019-2021).
//
// Options follow the reference's letters where they exist:
//   -r TASK     pagerank_double | pagerank | pagerank_double_push |
//               bfs_count | sssp_unweighted |
//               sssp_weighted | tc_u | tarjan_scc | bc_random | ppr
//   -R ROOT     root vertex (default 0)
//   -n N        iterations (PageRank, PPR; default 10)
//   -l N        load only the first N files (levels)
//   -c N        run the task N times (times each run)
//   -o FILE     write per-vertex results (first 50 vertices, like
//               print_results_part, benchmark.h:566-647); "-" = stdout
//   -k K        sources for bc_random / seeds for ppr (default 100 / 32)
//   -s SEED     seed for drawing sources (default 1)
//   -G SPEC     generate instead of reading files: rmat:SCALE:LEVELS:SEED
//   -d DEV      CUDA device (default 0)
#include <getopt.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include <algorithm>
#include <random>
#include <string>
#include <vector>

#include "lg.h"
#include "lg_host.h"

namespace {

double now_ms() {
	timespec ts;
	clock_gettime(CLOCK_MONOTONIC, &ts);
	return ts.tv_sec * 1e3 + ts.tv_nsec * 1e-6;
}

void die(const char* what, lg_status st) {
	char msg[512];
	lg_last_error(msg, sizeof msg);
	fprintf(stderr, "%s failed: %s (%s)\n", what, lg_status_string(st), msg);
	exit(1);
}

#define CHECK(call, what) do { lg_status _s = (call); if (_s) die(what, _s); } while (0)

struct Level {
	std::vector<uint32_t> src, dst, w, dsrc, ddst;
	bool weighted = false;
};

bool read_level(const char* path, Level& lv, uint64_t& max_id) {
	FILE* f = fopen(path, "r");
	if (!f) { perror(path); return false; }
	char line[1024];
	while (fgets(line, sizeof line, f)) {
		char* p = line;
		while (*p == ' ' || *p == '\t') p++;
		if (*p == '#' || *p == '%' || *p == '\n' || *p == 0) continue;
		bool del = false;
		if (*p == '-') { del = true; p++; }
		char* e;
		unsigned long long a = strtoull(p, &e, 10);
		if (e == p) continue;
		p = e;
		unsigned long long b = strtoull(p, &e, 10);
		if (e == p) continue;
		p = e;
		unsigned long long w = strtoull(p, &e, 10);
		bool has_w = e != p;
		max_id = std::max<uint64_t>(max_id, std::max(a, b));
		if (del) { lv.dsrc.push_back((uint32_t)a); lv.ddst.push_back((uint32_t)b); }
		else {
			lv.src.push_back((uint32_t)a);
			lv.dst.push_back((uint32_t)b);
			lv.w.push_back(has_w ? (uint32_t)w : 1u);
			lv.weighted |= has_w;
		}
	}
	fclose(f);
	return true;
}

void usage() {
	fprintf(stderr,
		"Usage: lg_benchmark [-r TASK] [-R ROOT] [-n ITERS] [-l LEVELS] [-c COUNT]\n"
		"                    [-o FILE] [-k K] [-s SEED] [-d DEV] [-N MAX_NODES]\n"
		"                    (-G rmat:S:L:SEED | FILE...)\n"
		"-N: vertices of the store (at least the largest id in the files + 1; the\n"
		"    reference's max_nodes, which PageRank's N counts)\n"
		"Tasks: pagerank_double pagerank pagerank_double_push bfs_count sssp_unweighted\n"
		"       sssp_weighted tc_u tarjan_scc bc_random ppr\n");
}

template <class T>
void print_part(FILE* f, const T* x, uint64_t V, const char* fmt) {
	for (uint64_t n = 0; n < V && n < 50; n++) {
		fprintf(f, "%llu\t", (unsigned long long)n);
		fprintf(f, fmt, x[n]);
		fprintf(f, "\n");
	}
}

} // namespace

int main(int argc, char** argv) {
	std::string task = "pagerank_double", out_file, gen;
	long long root = 0;
	int iters = 10, max_levels = -1, count = 1, device = 0, k = -1;
	unsigned long long min_nodes = 0;
	unsigned seed = 1;
	int c;
	while ((c = getopt(argc, argv, "r:R:n:l:c:o:k:s:G:d:N:h")) != -1) {
		switch (c) {
		case 'r': task = optarg; break;
		case 'R': root = atoll(optarg); break;
		case 'n': iters = atoi(optarg); break;
		case 'l': max_levels = atoi(optarg); break;
		case 'c': count = atoi(optarg); break;
		case 'o': out_file = optarg; break;
		case 'k': k = atoi(optarg); break;
		case 's': seed = (unsigned)atoi(optarg); break;
		case 'G': gen = optarg; break;
		case 'd': device = atoi(optarg); break;
		case 'N': min_nodes = strtoull(optarg, nullptr, 10); break;
		default: usage(); return c == 'h' ? 0 : 1;
		}
	}
	std::vector<std::string> files(argv + optind, argv + argc);
	if (files.empty() && gen.empty()) { usage(); return 1; }

	// ---- load: one file (or generated level) per level ----
	double t0 = now_ms();
	lg_hgraph* g = nullptr;
	bool weighted = false;
	if (!gen.empty()) {
		lg_graph_spec s;
		memset(&s, 0, sizeof s);
		int scale = 0, levels = 1;
		unsigned long long gs = 1;
		if (sscanf(gen.c_str(), "rmat:%d:%d:%llu", &scale, &levels, &gs) < 1) { usage(); return 1; }
		s.kind = LG_GEN_RMAT; s.scale = scale; s.edge_factor = 16; s.a = 0.57; s.b = 0.19;
		s.c = 0.19; s.seed = gs; s.num_levels = levels; s.level0_fraction = levels > 1 ? 0.9 : 1.0;
		s.delete_fraction = levels > 1 ? 0.002 : 0.0; s.split_seed = gs * 1000 + 17;
		s.weight_max = 255; s.weight_seed = gs * 1000 + 29;
		CHECK(lg_hgraph_create(&g, 1ull << scale, 1), "lg_hgraph_create");
		CHECK(lg_hgraph_build(g, &s), "lg_hgraph_build");
		weighted = true;
	} else {
		if (max_levels > 0 && (size_t)max_levels < files.size()) files.resize(max_levels);
		std::vector<Level> lv(files.size());
		uint64_t max_id = 0;
		for (size_t i = 0; i < files.size(); i++)
			if (!read_level(files[i].c_str(), lv[i], max_id)) return 1;
		for (auto& l : lv) weighted |= l.weighted;
		CHECK(lg_hgraph_create(&g, std::max<uint64_t>(max_id + 1, min_nodes), 1),
				"lg_hgraph_create");
		for (auto& l : lv)
			CHECK(lg_hgraph_add_level(g, l.src.data(), l.dst.data(), l.src.size(),
					l.dsrc.data(), l.ddst.data(), l.dsrc.size(),
					weighted ? l.w.data() : nullptr), "lg_hgraph_add_level");
	}
	const uint64_t V = lg_hgraph_max_nodes(g);
	lg_store* store = nullptr;
	lg_store_opts o = {device, nullptr, 1, 0};
	CHECK(lg_store_create(&store, &o), "lg_store_create");
	CHECK(lg_hgraph_ingest(g, store, 0), "lg_hgraph_ingest");
	lg_snapshot* snap = nullptr;
	CHECK(lg_snapshot_open(store, -1, &snap), "lg_snapshot_open");
	uint64_t E = 0;
	lg_snapshot_num_edges(snap, &E);
	printf("Loaded %d level(s): %llu vertices, %llu live edges (%.1f ms)\n",
			lg_store_num_levels(store), (unsigned long long)V, (unsigned long long)E,
			now_ms() - t0);

	// sources for bc_random / ppr: vertices with out-edges, seeded
	std::vector<uint32_t> deg(V);
	lg_out_degrees(snap, deg.data());
	auto draw = [&](int n) {
		std::vector<int64_t> cand, out;
		for (uint64_t v = 0; v < V; v++) if (deg[v]) cand.push_back((int64_t)v);
		std::mt19937_64 rng(seed);
		for (int i = 0; i < n && !cand.empty(); i++) out.push_back(cand[rng() % cand.size()]);
		return out;
	};

	double ret = NAN;
	FILE* of = nullptr;
	if (!out_file.empty()) of = out_file == "-" ? stdout : fopen(out_file.c_str(), "w");
	for (int run = 0; run < count; run++) {
		double ts = now_ms();
		if (task == "pagerank_double" || task == "pagerank") {
			std::vector<double> pr(V);
			// the reference's do-while loop runs one iteration for -n 0
			CHECK(lg_pagerank_pull(snap, std::max(iters, 1), 0.85, pr.data()),
					"lg_pagerank_pull");
			double s = 0;
			for (double x : pr) s += x;
			ret = s;
			if (of && run == count - 1) print_part(of, pr.data(), V, "%0.6lf");
		} else if (task == "pagerank_double_push") {
			std::vector<double> pr(V);
			CHECK(lg_pagerank_push(snap, std::max(iters, 1), 0.85, pr.data()),
					"lg_pagerank_push");
			double s = 0;
			for (double x : pr) s += x;
			ret = s;
			if (of && run == count - 1) print_part(of, pr.data(), V, "%0.6lf");
		} else if (task == "bfs_count" || task == "sssp_unweighted") {
			std::vector<int32_t> lvl(V);
			lg_bfs_result r;
			CHECK(lg_bfs(snap, root, lvl.data(), &r), "lg_bfs");
			ret = (double)r.reached;
			if (of && run == count - 1) print_part(of, lvl.data(), V, "%d");
		} else if (task == "sssp_weighted") {
			if (!weighted) { fprintf(stderr, "sssp_weighted needs weights (3rd column)\n"); return 1; }
			std::vector<uint32_t> dist(V);
			lg_sssp_result r;
			CHECK(lg_sssp_delta(snap, root, 32, dist.data(), &r), "lg_sssp_delta");
			ret = (double)r.reached;
			if (of && run == count - 1) print_part(of, dist.data(), V, "%u");
		} else if (task == "tc_u") {
			lg_tc_result r;
			CHECK(lg_triangle_count(snap, &r), "lg_triangle_count");
			ret = (double)r.triangles;
		} else if (task == "tarjan_scc") {
			std::vector<int64_t> lab(V);
			lg_scc_result r;
			CHECK(lg_scc(snap, lab.data(), &r), "lg_scc");
			ret = (double)r.components;        // true SCC count (the reference's
			                                   // value is the max of its labels)
			if (of && run == count - 1) print_part(of, lab.data(), V, "%lld");
		} else if (task == "bc_random") {
			auto src = draw(k > 0 ? k : 100);
			std::vector<double> bc(V);
			CHECK(lg_bc_batched(snap, src.data(), (int)src.size(), bc.data()), "lg_bc_batched");
			double m = 0;
			for (double x : bc) m = std::max(m, x);
			ret = m;                           // finalize() returns the max (bc_random.h:201-209)
			if (of && run == count - 1) print_part(of, bc.data(), V, "%0.6lf");
		} else if (task == "ppr") {
			const int K = k > 0 ? k : 32;
			auto sd = draw(K);
			std::vector<double> x(V * (size_t)K);
			CHECK(lg_ppr(&snap, 1, sd.data(), K, iters, 0.85, x.data()), "lg_ppr");
			double s = 0;
			for (double v : x) s += v;
			ret = s / K;
		} else {
			fprintf(stderr, "unknown task %s\n", task.c_str());
			usage();
			return 1;
		}
		printf("Run %d: %.3f ms\n", run + 1, now_ms() - ts);
	}
	if (of && of != stdout) fclose(of);
	if (!isnan(ret)) printf("Return value: %lf\n", ret);
	lg_snapshot_close(snap);
	lg_store_destroy(store);
	lg_hgraph_destroy(g);
	return 0;
}
