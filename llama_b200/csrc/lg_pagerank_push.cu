// lg_pagerank_push.cu - PageRank, push direction, FP64.
//
// Reference: ll_b_pagerank_push_ext<Graph,double>::run
// (benchmark/benchmarks/pagerank.h:258-318): pr0 = 1/N (N = max_nodes); per
// iteration every vertex t with out-degree > 0 adds pr[t] / out_degree(t) to
// nxt[w] for each out-neighbour w (an FP compare-and-swap ATOMIC_ADD,
// ll_utils.h:546-555), then pr[t] = (1-d)/N + d * nxt[t] and nxt[t] = 0.
//
// It reads only the out-CSR, so it runs on stores kept without reverse edges,
// where the pull variant cannot.  Here the out-edges are walked in balanced
// 1024-slot ranges (lg_expand.cuh), a warp per range: contrib[t] =
// pr[t] / out_degree(t) is computed once per vertex by the finishing kernel of
// the previous iteration, and each live edge issues one FP64 reduction
// (red.global.add.f64) on nxt[w].  Like the reference, the order in which a
// vertex's terms are added depends on the schedule, so results agree with
// the pull variant within FP64 rounding, not bit for bit.  A flattened
// out-CSR (lg_snapshot_flatten(snap, 0)) is read through its one-fragment
// view when present.
#include "lg_expand.cuh"
#include "lg_flat.cuh"

namespace lg {

constexpr uint32_t kPushRange = 1024;   // slots per warp range
constexpr int kPushThreads = 256;

// contrib[t] = pr0 / out_degree(t) (0 without out-edges), nxt[t] = 0.
__global__ void push_init(const uint32_t* outdeg, uint64_t V, double pr0, double* contrib,
		double* nxt, double* pr_out) {
	const uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (v >= V) return;
	const uint32_t dg = __ldg(outdeg + v);
	contrib[v] = dg ? pr0 / (double)dg : 0.0;
	nxt[v] = 0.0;
	if (pr_out) pr_out[v] = pr0;
}

// Every live out-edge t -> w adds contrib[t] to nxt[w].
__global__ void __launch_bounds__(kPushThreads)
push_scatter(SnapCsr out, const uint32_t* pos, uint32_t total, uint32_t V,
		const double* contrib, double* nxt) {
	const uint32_t nranges = (total + kPushRange - 1) / kPushRange;
	const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
	for (uint32_t r = warp; r < nranges; r += nwarps) {
		range_for_each(out, nullptr, pos, V, total, nranges, kPushRange, r,
			[&](bool act, uint32_t, uint32_t t, uint32_t w, uint32_t, uint32_t) {
				if (act) {
					const double c = __ldg(contrib + t);
					if (c != 0.0) atomicAdd(nxt + w, c);
				}
			});
	}
}

// pr[t] = (1-d)/N + d * nxt[t]; the next contrib; nxt cleared for the next
// scatter.  pr_out is written on the last iteration only.
__global__ void push_finish(const uint32_t* outdeg, uint64_t V, double base, double d,
		double* nxt, double* contrib, double* pr_out) {
	const uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (v >= V) return;
	const double pr = __dadd_rn(base, __dmul_rn(d, nxt[v]));
	nxt[v] = 0.0;
	const uint32_t dg = __ldg(outdeg + v);
	contrib[v] = dg ? pr / (double)dg : 0.0;
	if (pr_out) pr_out[v] = pr;
}

} // namespace lg

using namespace lg;

extern "C" lg_status lg_pagerank_push(lg_snapshot* sn, int iterations, double damping,
		double* ranks) {
	clear_error();
	if (!sn || !ranks) return set_error(LG_EINVAL, "null argument");
	if (!(damping > 0.0 && damping < 1.0))
		return set_error(LG_EINVAL, "damping must be in (0, 1)");
	if (iterations < 0) return set_error(LG_EINVAL, "iterations must be >= 0");
	lg_store* s = sn->store;
	LG_CUDA(cudaSetDevice(s->device), "cudaSetDevice");
	cudaStream_t st = s->stream;
	const uint64_t V = sn->V;
	if (V == 0) return LG_OK;
	const double N = (double)V;
	const double base = (1.0 - damping) / N;
	const unsigned B = 256;
	DevBuf* sc = s->scratch;
	const uint32_t* outdeg = sn->out.deg.as<uint32_t>();

	// the out-edges: the flat view when the snapshot has one, else the levels
	const FlatCsr* fo = sn->flat[0];
	const bool flat = fo && fo->has_view;
	const SnapCsr out = flat ? fo->view(outdeg) : sn->view(0);
	const uint32_t* pos = flat ? fo->off.as<uint32_t>() : sn->out.slot_off.as<uint32_t>();
	const uint32_t total = (uint32_t)(flat ? fo->E : sn->out.n_frag_slots);

	LG_TRY(sc[0].reserve(V * sizeof(double)));      // contrib
	LG_TRY(sc[1].reserve(V * sizeof(double)));      // nxt
	const bool dev_out = is_device_pointer(ranks);
	double* pr_buf = ranks;
	if (!dev_out) {
		LG_TRY(sc[4].reserve(V * sizeof(double)));
		pr_buf = sc[4].as<double>();
	}
	double* contrib = sc[0].as<double>();
	double* nxt = sc[1].as<double>();
	int sms = 148;
	cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->device);
	const unsigned scatter_blocks = (unsigned)sms * 8u;   // persistent over the ranges

	push_init<<<grid_for(V, B), B, 0, st>>>(outdeg, V, 1.0 / N, contrib, nxt,
			iterations == 0 ? pr_buf : nullptr);
	s->launches++;
	for (int it = 0; it < iterations; it++) {
		if (total > 0) {
			push_scatter<<<scatter_blocks, kPushThreads, 0, st>>>(out, pos, total,
					(uint32_t)V, contrib, nxt);
			s->launches++;
		}
		push_finish<<<grid_for(V, B), B, 0, st>>>(outdeg, V, base, damping, nxt, contrib,
				it == iterations - 1 ? pr_buf : nullptr);
		s->launches++;
	}
	LG_CUDA(cudaGetLastError(), "pagerank push");
	if (!dev_out) {
		LG_TRY(copy_out(s, ranks, pr_buf, V * sizeof(double)));
		LG_CUDA(cudaStreamSynchronize(st), "pagerank push");
	}
	return LG_OK;
}
