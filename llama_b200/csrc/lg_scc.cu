// lg_scc.cu - strongly connected components of a snapshot.
//
// Reference task: "tarjan_scc" (ll_b_tarjan_scc, benchmark/benchmarks/
// tarjan_scc.h:121-206).  That Green-Marl Tarjan uses vertex ids as low-links
// and does not compute true SCCs, so the contract here is the true SCC
// partition with every component labelled by its smallest vertex id.
//
// Algorithm: trim + colouring (Orzan; Slota et al.):
//   0. vertices with live in- or out-degree 0 are their own component;
//   1. every remaining vertex starts with colour = its id and the smallest
//      colour is pushed along out-edges to a fixpoint (atomicMin, worklist),
//      so colour(v) = smallest remaining vertex that reaches v;
//   2. a vertex whose colour is its own id is the smallest of its component;
//      a backward traversal over in-edges, restricted to vertices of the same
//      colour, collects exactly that component, labelled with the colour;
//   3. collected vertices leave the remaining set and 1-2 repeat.
// Each round removes at least the component of the smallest remaining
// vertex, and labels do not depend on thread order.
#include "lg_device.cuh"
#include "lg_expand.cuh"
#include "lg_queue.cuh"

namespace lg {

constexpr uint32_t kNone = 0xffffffffu;
constexpr uint32_t kSccRange = 1024;
constexpr int kSccThreads = 256;

constexpr int kSccListThreads = 256;   // CTA size of the per-vertex list kernels

// Trim: vertices without live in- or out-edges are singletons; the others
// form the initial remaining list.  ctr[0] = remaining count.
__global__ void scc_trim(const uint32_t* outdeg, const uint32_t* indeg, uint64_t V,
		uint32_t* label, uint32_t* mark, uint32_t* stamp, uint32_t* rem,
		unsigned long long* ctr) {
	const uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	bool keep = false;
	if (v < V) {
		keep = outdeg[v] != 0 && indeg[v] != 0;
		label[v] = keep ? kNone : (uint32_t)v;
		mark[v] = 0;
		stamp[v] = 0;
	}
	block_push<kSccListThreads>(keep, (uint32_t)v, rem, ctr);
}

__global__ void scc_color_init(const uint32_t* rem, uint32_t n, uint32_t* color) {
	const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n) { const uint32_t v = rem[i]; color[v] = v; }
}

// Forward colour propagation from worklist `wl` over out-edges.
__global__ void __launch_bounds__(kSccThreads)
scc_propagate(SnapCsr out, const uint32_t* wl, const uint32_t* pos, uint32_t n,
		uint32_t total, uint32_t nranges, const uint32_t* label, uint32_t* color,
		uint32_t* stamp, uint32_t round, uint32_t* next, unsigned long long* ctr) {
	__shared__ uint32_t sbuf[kSccThreads / 32][kPushBuf];
	const uint64_t r = (uint64_t)blockIdx.x * (kSccThreads / 32) + (threadIdx.x >> 5);
	if (r >= nranges) return;
	uint32_t* sb = sbuf[threadIdx.x >> 5];
	uint32_t nb = 0;
	range_for_each(out, wl, pos, n, total, nranges, kSccRange, (uint32_t)r,
		[&](bool act, uint32_t own, uint32_t v, uint32_t w, uint32_t, uint32_t) {
			bool push = false;
			if (act && __ldcg(label + w) == kNone) {
				const uint32_t c = __ldcg(color + v);
				if (c < __ldcg(color + w)) {
					const uint32_t old = atomicMin(color + w, c);
					if (c < old) push = atomicExch(stamp + w, round) != round;
				}
			}
			wq_add(push, w, sb, nb, next, ctr);
		});
	wq_flush(sb, nb, next, ctr);
}

// Roots: remaining vertices whose colour is their own id start the backward
// traversal of their component.
__global__ void scc_roots(const uint32_t* rem, uint32_t n, const uint32_t* color,
		uint32_t* mark, uint32_t round, uint32_t* frontier, unsigned long long* ctr) {
	const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	bool root = false;
	uint32_t v = 0;
	if (i < n) {
		v = rem[i];
		root = color[v] == v;
		if (root) mark[v] = round;
	}
	block_push<kSccListThreads>(root, v, frontier, ctr);
}

// Backward traversal over in-edges within a colour.
__global__ void __launch_bounds__(kSccThreads)
scc_backward(SnapCsr in, const uint32_t* fr, const uint32_t* pos, uint32_t n,
		uint32_t total, uint32_t nranges, const uint32_t* label, const uint32_t* color,
		uint32_t* mark, uint32_t round, uint32_t* next, unsigned long long* ctr) {
	__shared__ uint32_t sbuf[kSccThreads / 32][kPushBuf];
	const uint64_t r = (uint64_t)blockIdx.x * (kSccThreads / 32) + (threadIdx.x >> 5);
	if (r >= nranges) return;
	uint32_t* sb = sbuf[threadIdx.x >> 5];
	uint32_t nb = 0;
	range_for_each(in, fr, pos, n, total, nranges, kSccRange, (uint32_t)r,
		[&](bool act, uint32_t own, uint32_t v, uint32_t u, uint32_t, uint32_t) {
			bool push = false;
			if (act && __ldcg(label + u) == kNone && __ldcg(mark + u) != round
					&& __ldcg(color + u) == __ldcg(color + v))
				push = atomicExch(mark + u, round) != round;
			wq_add(push, u, sb, nb, next, ctr);
		});
	wq_flush(sb, nb, next, ctr);
}

// Collected vertices get their label; the rest stay for the next round.
__global__ void scc_collect(const uint32_t* rem, uint32_t n, const uint32_t* color,
		const uint32_t* mark, uint32_t round, uint32_t* label, uint32_t* rem_next,
		unsigned long long* ctr) {
	const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	bool keep = false;
	uint32_t v = 0;
	if (i < n) {
		v = rem[i];
		if (mark[v] == round) label[v] = color[v];
		else keep = true;
	}
	block_push<kSccListThreads>(keep, v, rem_next, ctr);
}

__global__ void scc_output(const uint32_t* label, uint64_t V, long long* out,
		unsigned long long* comps) {
	const uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	bool head = false;
	if (v < V) {
		out[v] = (long long)label[v];
		head = label[v] == (uint32_t)v;
	}
	// one counter atomic per CTA (kSccListThreads threads)
	__shared__ unsigned int s_heads;
	if (threadIdx.x == 0) s_heads = 0;
	__syncthreads();
	const unsigned m = __ballot_sync(0xffffffffu, head);
	if ((threadIdx.x & 31) == 0 && m) atomicAdd(&s_heads, (unsigned int)__popc(m));
	__syncthreads();
	if (threadIdx.x == 0 && s_heads) atomicAdd(comps, (unsigned long long)s_heads);
}

} // namespace lg

using namespace lg;

namespace {

// Expand `list` (n entries) over `g` with one of the range kernels; returns
// the size of the list the kernel appended to.
template <class Launch>
lg_status run_list_step(lg_store* s, const SnapCsr& g, const uint32_t* list, uint32_t n,
		DevBuf& cnt, DevBuf& pos, DevBuf& scan_tmp, unsigned long long* ctr,
		Launch&& launch, uint64_t* produced) {
	cudaStream_t st = s->stream;
	list_slots<<<grid_for(n, 256), 256, 0, st>>>(g, list, n, cnt.as<uint32_t>());
	uint64_t total = 0;
	LG_TRY(exclusive_scan_u32(cnt.as<uint32_t>(), pos.as<uint32_t>(), n, scan_tmp, st, &total));
	LG_CUDA(cudaMemsetAsync(ctr, 0, sizeof(unsigned long long), st), "memset");
	const uint32_t nranges = (uint32_t)((total + kSccRange - 1) / kSccRange);
	if (nranges) launch(grid_for(nranges, kSccThreads / 32), (uint32_t)total, nranges);
	LG_CUDA(cudaGetLastError(), "scc step");
	s->launches += 4 + (nranges ? 1 : 0);
	unsigned long long h = 0;
	LG_TRY(read_words(s, ctr, 1, &h));
	*produced = h;
	return LG_OK;
}

lg_status read_ctr(lg_store* s, unsigned long long* ctr, uint64_t* v) {
	unsigned long long h = 0;
	LG_TRY(read_words(s, ctr, 1, &h));
	*v = h;
	return LG_OK;
}

} // namespace

extern "C" lg_status lg_scc(lg_snapshot* sn, int64_t* labels, lg_scc_result* result) {
	clear_error();
	if (!sn || !labels) return set_error(LG_EINVAL, "null argument");
	if (!sn->in.present) return set_error(LG_ESTATE, "SCC needs the in-CSR (reverse edges)");
	lg_store* s = sn->store;
	LG_CUDA(cudaSetDevice(s->device), "cudaSetDevice");
	cudaStream_t st = s->stream;
	const uint64_t V = sn->V;
	DevBuf label, color, mark, stamp, rem, rem2, wl, wl2, cnt, pos, scan_tmp, ctrb, outb;
	for (DevBuf* b : {&label, &color, &mark, &stamp, &rem, &rem2, &wl, &wl2, &cnt})
		LG_TRY(b->reserve(V * 4));
	LG_TRY(pos.reserve((V + 1) * 4));
	LG_TRY(ctrb.reserve(2 * sizeof(unsigned long long)));
	unsigned long long* ctr = ctrb.as<unsigned long long>();
	const SnapCsr out = sn->view(0), in = sn->view(1);
	uint32_t* lab = label.as<uint32_t>();
	uint32_t* col = color.as<uint32_t>();
	uint32_t* mk = mark.as<uint32_t>();
	uint32_t* stp = stamp.as<uint32_t>();

	LG_CUDA(cudaMemsetAsync(ctr, 0, sizeof(unsigned long long), st), "memset");
	scc_trim<<<grid_for(V, kSccListThreads), kSccListThreads, 0, st>>>(sn->out.deg.as<uint32_t>(),
			sn->in.deg.as<uint32_t>(), V, lab, mk, stp, rem.as<uint32_t>(), ctr);
	LG_CUDA(cudaGetLastError(), "scc_trim");
	s->launches++;
	uint64_t n_rem = 0;
	LG_TRY(read_ctr(s, ctr, &n_rem));
	const uint64_t trimmed = V - n_rem;
	uint32_t round = 0, prop_round = 0;
	int steps = 0;
	uint32_t* R = rem.as<uint32_t>();
	uint32_t* R2 = rem2.as<uint32_t>();
	while (n_rem > 0) {
		round++;
		if (round > V + 1) return set_error(LG_ETIMEOUT, "SCC did not converge");
		scc_color_init<<<grid_for(n_rem, 256), 256, 0, st>>>(R, (uint32_t)n_rem, col);
		LG_CUDA(cudaMemcpyAsync(wl.p, R, n_rem * 4, cudaMemcpyDeviceToDevice, st), "d2d");
		s->launches++;
		uint32_t* W = wl.as<uint32_t>();
		uint32_t* W2 = wl2.as<uint32_t>();
		uint64_t nw = n_rem;
		while (nw > 0) {
			prop_round++;
			uint64_t produced = 0;
			LG_TRY(run_list_step(s, out, W, (uint32_t)nw, cnt, pos, scan_tmp, ctr,
				[&](unsigned blocks, uint32_t total, uint32_t nranges) {
					scc_propagate<<<blocks, kSccThreads, 0, st>>>(out, W, pos.as<uint32_t>(),
							(uint32_t)nw, total, nranges, lab, col, stp, prop_round, W2, ctr);
				}, &produced));
			std::swap(W, W2);
			nw = produced;
			steps++;
		}
		// backward traversal from the roots
		LG_CUDA(cudaMemsetAsync(ctr, 0, sizeof(unsigned long long), st), "memset");
		scc_roots<<<grid_for(n_rem, kSccListThreads), kSccListThreads, 0, st>>>(R, (uint32_t)n_rem, col, mk, round,
				W, ctr);
		LG_CUDA(cudaGetLastError(), "scc_roots");
		s->launches++;
		uint64_t nf = 0;
		LG_TRY(read_ctr(s, ctr, &nf));
		while (nf > 0) {
			uint64_t produced = 0;
			LG_TRY(run_list_step(s, in, W, (uint32_t)nf, cnt, pos, scan_tmp, ctr,
				[&](unsigned blocks, uint32_t total, uint32_t nranges) {
					scc_backward<<<blocks, kSccThreads, 0, st>>>(in, W, pos.as<uint32_t>(),
							(uint32_t)nf, total, nranges, lab, col, mk, round, W2, ctr);
				}, &produced));
			std::swap(W, W2);
			nf = produced;
			steps++;
		}
		LG_CUDA(cudaMemsetAsync(ctr, 0, sizeof(unsigned long long), st), "memset");
		scc_collect<<<grid_for(n_rem, kSccListThreads), kSccListThreads, 0, st>>>(R, (uint32_t)n_rem, col, mk, round,
				lab, R2, ctr);
		LG_CUDA(cudaGetLastError(), "scc_collect");
		s->launches++;
		uint64_t left = 0;
		LG_TRY(read_ctr(s, ctr, &left));
		if (left >= n_rem) return set_error(LG_ECUDA, "SCC round made no progress");
		n_rem = left;
		std::swap(R, R2);
	}
	const bool dev_out = is_device_pointer(labels);
	long long* o = (long long*)labels;
	if (!dev_out) { LG_TRY(outb.reserve(V * 8)); o = outb.as<long long>(); }
	LG_CUDA(cudaMemsetAsync(ctr + 1, 0, sizeof(unsigned long long), st), "memset");
	scc_output<<<grid_for(V, kSccListThreads), kSccListThreads, 0, st>>>(lab, V, o, ctr + 1);
	LG_CUDA(cudaGetLastError(), "scc_output");
	s->launches++;
	uint64_t comps = 0;
	LG_TRY(read_ctr(s, ctr + 1, &comps));
	if (!dev_out) {
		LG_TRY(copy_out(s, labels, o, V * 8));
		LG_CUDA(cudaStreamSynchronize(st), "scc");
	}
	if (result) {
		result->components = comps;
		result->trimmed = trimmed;
		result->rounds = (int32_t)round;
		result->steps = steps;
	}
	return LG_OK;
}
