// lg_adjoint.cu - weighted PageRank to a fixed point and its adjoint.
//
// No reference counterpart: the forward is the pull iteration of
// ll_b_pagerank_pull_ext::run (benchmark/benchmarks/pagerank.h:120-169)
// with per-edge weights P(w->t) and a teleport vector v,
//     x = (1-d) v + d P^T x                                     (forward)
// iterated from x = v until sum |x' - x| < tol.  The backward differentiates
// the fixed point implicitly: with g = dL/dx,
//     lambda = g + d P lambda                                   (adjoint)
// iterated the same way over OUT-edges, then
//     dL/dv = (1-d) lambda,   dL/dP(w->t) = d lambda[t] x[w].
// Only the converged x is kept between the two calls (the "tape"), no
// iterate is stored.
//
// Edge weights and their gradients are indexed by the snapshot's
// out-adjacency order (the order lg_snapshot_adjacency(dir 0) returns).  On
// first use a snapshot gets its live adjacency flattened in both directions
// (lg_flat.cuh) and a map from every flat in-edge to its out-adjacency
// position; the flat out-CSR lists the edges in exactly that order, so the
// backward sweep reads the weights as given and the forward gathers them
// once per call into in-edge order.
//
// Both sweeps are the flat sweep of lg_flat_sweep.cuh with an affine op:
// y[v] = base[v] + d * sum over v's edges k of w[k] * x[nbr(k)], and the
// residual sum |y - x| accumulated per iteration in device memory.  The
// host does not wait for every iteration: it issues iterations in chunks,
// every launch first reads the previous iteration's residual and does
// nothing once it is below tol, and the host reads the residuals of a chunk
// while the next one runs.  The result is the one the stop-at-first-
// residual-below-tol loop gives, with no synchronisation per iteration.
#include "lg_flat_sweep.cuh"
#include "lg_tune.h"

#include <cmath>

namespace lg {

constexpr uint32_t kNoPos = 0xffffffffu;
constexpr int kChunk = 16;            // iterations issued between residual reads

// One iteration of y = base + d * (weighted pull of x) over a flat CSR.
struct AffOp {
	static constexpr bool kResidual = true;
	const uint32_t* nz_rows;   // R
	const double* w;           // E, in the flat CSR's edge order
	const double* x;
	const double* base;
	double* y;
	double* resid;             // this iteration's sum |y - x|
	const double* prev;        // the previous iteration's, null for the first
	double d, tol;
	uint32_t E;
	__device__ __forceinline__ bool skip() const { return prev && __ldcg(prev) < tol; }
	__device__ __forceinline__ void values(uint32_t eb, const uint32_t (&id)[kFlatPerLane],
			double (&v)[kFlatPerLane]) const {
		double wv[kFlatPerLane];
		if (eb + kFlatPerLane <= E) {
			// two 32-byte loads (eb is a multiple of 8), streamed
			asm("ld.global.cs.v4.f64 {%0, %1, %2, %3}, [%4];"
				: "=d"(wv[0]), "=d"(wv[1]), "=d"(wv[2]), "=d"(wv[3]) : "l"(w + eb));
			asm("ld.global.cs.v4.f64 {%0, %1, %2, %3}, [%4];"
				: "=d"(wv[4]), "=d"(wv[5]), "=d"(wv[6]), "=d"(wv[7]) : "l"(w + eb + 4));
		} else {
#pragma unroll
			for (int i = 0; i < kFlatPerLane; i++) wv[i] = eb + i < E ? __ldcs(w + eb + i) : 0.0;
		}
#pragma unroll
		for (int i = 0; i < kFlatPerLane; i++)
			v[i] = id[i] != kNoId ? __dmul_rn(wv[i], __ldg(x + id[i])) : 0.0;
	}
	__device__ __forceinline__ double finish(uint32_t k, double s) const {
		const uint32_t v = __ldg(nz_rows + k);
		const double yv = __dadd_rn(__ldg(base + v), __dmul_rn(d, s));
		y[v] = yv;
		return fabs(yv - __ldg(x + v));
	}
	__device__ __forceinline__ void residual(double r) const { atomicAdd(resid, r); }
};

__global__ void __launch_bounds__(kFlatWarps * 32)
aff_flat_step(FlatTiles a, AffOp op) {
	__shared__ double rowsum[kFlatWarps][kFlatTile];
	flat_sweep_tile(a, op, rowsum);
}

template <int kMinBlocks>
__global__ void __launch_bounds__(kFlatLoopWarps * 32, kMinBlocks)
aff_flat_loop(FlatTiles a, AffOp op) {
	__shared__ double rowsum[kFlatLoopWarps][kFlatTile];
	flat_sweep_loop(a, op, rowsum);
}

__global__ void __launch_bounds__(kFixupThreads)
aff_flat_fixup(FlatTiles a, AffOp op) {
	flat_sweep_fixup_body(a, op);
}

// Rows without edges: y[v] = base[v] in every iteration.  Written into y
// with their first-iteration residual |base - x0| added to resid0, or (resid0
// null) just written.
__global__ void aff_empty_rows(const uint32_t* off, uint64_t V, const double* base,
		const double* x0, double* y, double* resid0) {
	const uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	double r = 0.0;
	if (v < V && __ldg(off + v + 1) == __ldg(off + v)) {
		const double b = __ldg(base + v);
		y[v] = b;
		if (resid0) r = fabs(b - __ldg(x0 + v));
	}
	if (!resid0) return;
#pragma unroll
	for (int o = 16; o > 0; o >>= 1) r += __shfl_xor_sync(0xffffffffu, r, o);
	if ((threadIdx.x & 31u) == 0 && r != 0.0) atomicAdd(resid0, r);
}

// --- per-snapshot maps ----------------------------------------------------

// out_pos[k] for every out-CSR virtual slot k: position of the live edge in
// the out-adjacency order (kNoPos for deleted slots); also src/dst per
// position.  One thread per vertex, walking its chain.
__global__ void adj_out_map(SnapCsr g, const uint32_t* slot_off, const uint64_t* adj_off,
		uint32_t* out_pos, uint32_t* src, uint32_t* dst, uint32_t* bad) {
	const uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (v >= g.V) return;
	const LevelTab* lt = g.lt;
	uint64_t p = adj_off[v];
	uint32_t k = slot_off[v];
	for (uint32_t f = g.frag_off[v]; f < g.frag_off[v + 1]; f++) {
		const uint2 fr = g.frags[f];
		const uint32_t lv = frag_level(fr);
		for (uint32_t i = 0; i < frag_len(fr); i++, k++) {
			const uint32_t idx = fr.x + i;
			if (slot_deleted(lt, lv, idx)) { out_pos[k] = kNoPos; continue; }
			out_pos[k] = (uint32_t)p;
			src[p] = (uint32_t)v;
			dst[p] = lt->ids[lv][idx];
			p++;
		}
	}
	if (p != adj_off[v + 1]) atomicOr(bad, 1u);
}

// in_pos[q] for every in-CSR virtual slot q of vertex t holding source w:
// the out-adjacency position of edge (w -> t), found by binary search in
// w's out-fragments (each sorted by target id).
__global__ void adj_in_map(SnapCsr in, const uint32_t* in_slot_off, SnapCsr out,
		const uint32_t* out_slot_off, const uint32_t* out_pos, uint32_t* in_pos,
		uint32_t* bad) {
	const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= in.V) return;
	uint32_t q = in_slot_off[t];
	for (uint32_t f = in.frag_off[t]; f < in.frag_off[t + 1]; f++) {
		const uint2 fr = in.frags[f];
		const uint32_t lv = frag_level(fr);
		for (uint32_t i = 0; i < frag_len(fr); i++, q++) {
			const uint32_t idx = fr.x + i;
			if (slot_deleted(in.lt, lv, idx)) { in_pos[q] = kNoPos; continue; }
			const uint32_t w = in.lt->ids[lv][idx];
			uint32_t found = kNoPos, k = out_slot_off[w];
			for (uint32_t g2 = out.frag_off[w]; g2 < out.frag_off[w + 1] && found == kNoPos; g2++) {
				const uint2 of = out.frags[g2];
				const uint32_t* ids = out.lt->ids[frag_level(of)] + of.x;
				uint32_t lo = 0, hi = frag_len(of);
				while (lo < hi) {
					const uint32_t mid = (lo + hi) >> 1;
					if (ids[mid] < (uint32_t)t) lo = mid + 1; else hi = mid;
				}
				// the live copy of (w, t): skip deleted duplicates
				for (uint32_t j = lo; j < frag_len(of) && ids[j] == (uint32_t)t; j++)
					if (out_pos[k + j] != kNoPos) { found = out_pos[k + j]; break; }
				k += frag_len(of);
			}
			in_pos[q] = found;
			if (found == kNoPos) atomicOr(bad, 1u);
		}
	}
}

__global__ void gather_weights(const uint32_t* map, uint64_t n, const double* w,
		double* out) {
	const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n) { const uint32_t p = map[i]; out[i] = p == kNoPos ? 0.0 : w[p]; }
}

__global__ void scale_vec(const double* a, double s, uint64_t n, double* out) {
	const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n) out[i] = s * a[i];
}

__global__ void edge_grad(const uint32_t* src, const uint32_t* dst, uint64_t E, double d,
		const double* lam, const double* x, double* out) {
	const uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (p < E) out[p] = d * (lam[dst[p]] * x[src[p]]);
}

__global__ void widen_prefix(const uint32_t* p32, uint64_t n, uint64_t* p64) {
	const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i <= n) p64[i] = p32[i];
}

// 1 for the virtual in-slots that hold a live edge
__global__ void live_flags(const uint32_t* pos, uint64_t n, uint32_t* flag) {
	const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n) flag[i] = pos[i] != kNoPos;
}

// in_pos of the flat in-CSR: the live virtual slots' positions, compacted in
// slot order (the order in which the flat in-CSR lists them); each one's
// source must be the flat in-edge's id
__global__ void compact_in_pos(const uint32_t* pos, const uint32_t* at, uint64_t n,
		const uint32_t* src, const uint32_t* flat_ids, uint32_t* out, uint32_t* bad) {
	const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	const uint32_t p = pos[i];
	if (p == kNoPos) return;
	const uint32_t k = at[i];
	out[k] = p;
	if (src[p] != __ldg(flat_ids + k)) atomicOr(bad, 2u);
}

// the flat out-CSR must list the out-edges in out-adjacency order
__global__ void check_out_order(const uint32_t* dst, const uint32_t* flat_ids, uint64_t E,
		uint32_t* bad) {
	const uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (p < E && dst[p] != flat_ids[p]) atomicOr(bad, 4u);
}

} // namespace lg

using namespace lg;

struct lg_adjoint_maps {
	FlatCsr fin, fout;     // the snapshot's live adjacency, flat, per direction
	DevBuf in_pos;         // E u32: out-adjacency position of each flat in-edge
	DevBuf src;            // E u32: source of each out-adjacency position
	uint64_t E = 0;
	// solve buffers, reused by every call on the snapshot
	DevBuf xa, xb, base, win, carries, resid, stage_w, stage_v, stage_g;
	double* resid_host = nullptr;          // pinned, 2 * kChunk
	cudaEvent_t chunk_done[2] = {nullptr, nullptr};
	~lg_adjoint_maps() {
		if (resid_host) cudaFreeHost(resid_host);
		for (cudaEvent_t e : chunk_done) if (e) cudaEventDestroy(e);
	}
};

struct lg_adjoint {
	lg_snapshot* snap = nullptr;
	double d = 0.85, tol = 1e-12;
	int max_iter = 0;
	DevBuf x, w;           // converged scores; the weights, out-adjacency order
};

namespace {

lg_status build_maps(lg_snapshot* sn, lg_adjoint_maps* m) {
	lg_store* s = sn->store;
	cudaStream_t st = s->stream;
	const uint64_t V = sn->V;
	const uint64_t E = m->E;
	DevBuf out_pos, in_pos, dst, adj_off, p32, scan_tmp, badb, flag, at;
	LG_TRY(out_pos.reserve(std::max<uint64_t>(sn->out.n_frag_slots, 1) * 4));
	LG_TRY(in_pos.reserve(std::max<uint64_t>(sn->in.n_frag_slots, 1) * 4));
	LG_TRY(m->src.reserve(std::max<uint64_t>(E, 1) * 4));
	LG_TRY(dst.reserve(std::max<uint64_t>(E, 1) * 4));
	LG_TRY(adj_off.reserve((V + 1) * 8));
	LG_TRY(p32.reserve((V + 1) * 4));
	LG_TRY(badb.reserve(4));
	uint64_t tot = 0;
	LG_TRY(exclusive_scan_u32(sn->out.deg.as<uint32_t>(), p32.as<uint32_t>(), V, scan_tmp, st,
			&tot));
	if (tot != E) return set_error(LG_EINVAL, "out-degrees do not add up to the live edges");
	LG_CUDA(cudaMemsetAsync(badb.p, 0, 4, st), "memset");
	widen_prefix<<<grid_for(V + 1, 256), 256, 0, st>>>(p32.as<uint32_t>(), V,
			adj_off.as<uint64_t>());
	const SnapCsr out = sn->view(0), in = sn->view(1);
	adj_out_map<<<grid_for(V, 128), 128, 0, st>>>(out, sn->out.slot_off.as<uint32_t>(),
			adj_off.as<uint64_t>(), out_pos.as<uint32_t>(), m->src.as<uint32_t>(),
			dst.as<uint32_t>(), badb.as<uint32_t>());
	adj_in_map<<<grid_for(V, 128), 128, 0, st>>>(in, sn->in.slot_off.as<uint32_t>(), out,
			sn->out.slot_off.as<uint32_t>(), out_pos.as<uint32_t>(), in_pos.as<uint32_t>(),
			badb.as<uint32_t>());
	LG_CUDA(cudaGetLastError(), "adjoint maps");
	s->launches += 3;
	// flat CSRs of both directions; the in-edge map compacted to the flat order
	LG_TRY(build_flat(sn, 1, m->fin, false));
	LG_TRY(build_flat(sn, 0, m->fout, false));
	if (m->fin.E != E || m->fout.E != E)
		return set_error(LG_EINVAL, "the in- and out-CSR of the snapshot differ in edge count");
	const uint64_t n = sn->in.n_frag_slots;
	LG_TRY(flag.reserve(std::max<uint64_t>(n, 1) * 4));
	LG_TRY(at.reserve((n + 1) * 4));
	LG_TRY(m->in_pos.reserve(std::max<uint64_t>(E, 1) * 4));
	live_flags<<<grid_for(n, 256), 256, 0, st>>>(in_pos.as<uint32_t>(), n, flag.as<uint32_t>());
	LG_CUDA(cudaGetLastError(), "live flags");
	uint64_t live = 0;
	LG_TRY(exclusive_scan_u32(flag.as<uint32_t>(), at.as<uint32_t>(), n, scan_tmp, st, &live));
	if (live != E) return set_error(LG_EINVAL, "in-CSR live slots differ from the edge count");
	compact_in_pos<<<grid_for(n, 256), 256, 0, st>>>(in_pos.as<uint32_t>(), at.as<uint32_t>(),
			n, m->src.as<uint32_t>(), m->fin.ids.as<uint32_t>(), m->in_pos.as<uint32_t>(),
			badb.as<uint32_t>());
	check_out_order<<<grid_for(E, 256), 256, 0, st>>>(dst.as<uint32_t>(),
			m->fout.ids.as<uint32_t>(), E, badb.as<uint32_t>());
	s->launches += 4;
	uint32_t bad = 0;
	LG_CUDA(cudaGetLastError(), "adjoint maps");
	LG_CUDA(cudaMemcpyAsync(&bad, badb.p, 4, cudaMemcpyDeviceToHost, st), "d2h");
	LG_CUDA(cudaStreamSynchronize(st), "adjoint maps");
	if (bad)
		return set_error(LG_EINVAL, "out- and in-CSR of the snapshot disagree, or a "
				"fragment is not sorted by neighbour id (code %u)", bad);
	LG_CUDA(cudaHostAlloc((void**)&m->resid_host, 2 * kChunk * sizeof(double),
			cudaHostAllocDefault), "cudaHostAlloc");
	for (cudaEvent_t& e : m->chunk_done)
		LG_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate");
	return LG_OK;
}

lg_status ensure_maps(lg_snapshot* sn) {
	if (sn->adj_maps) return LG_OK;
	const uint64_t E = sn->out.n_edges;
	if (E > 0xffffffffull - 2 * kFlatTile)
		return set_error(LG_ENOTSUP, "more than 2^32 - %u live edges", 2 * kFlatTile);
	lg_adjoint_maps* m = new (std::nothrow) lg_adjoint_maps();
	if (!m) return set_error(LG_ENOMEM, "host allocation");
	m->E = E;
	lg_status r = build_maps(sn, m);
	if (r) { delete m; return r; }
	sn->adj_maps = m;
	return LG_OK;
}

// Iterate y = base + d * (weighted pull of x) over the flat CSR f until
// sum |y - x| < tol (at most max_iter iterations); m->xa holds the start on
// entry.  *out points at the result (m->xa or m->xb) on return.
lg_status fixed_point(lg_snapshot* sn, const FlatCsr& f, const double* w, const double* base,
		double d, double tol, int max_iter, int* iters, double* resid_out, double** out) {
	lg_store* s = sn->store;
	lg_adjoint_maps* m = sn->adj_maps;
	cudaStream_t st = s->stream;
	const uint64_t V = sn->V;
	double* A = m->xa.as<double>();
	double* B = m->xb.as<double>();
	LG_TRY(m->carries.reserve(2ull * std::max<uint32_t>(f.ntiles, 1) * sizeof(double)));
	LG_TRY(m->resid.reserve((size_t)max_iter * sizeof(double)));
	double* resid = m->resid.as<double>();
	LG_CUDA(cudaMemsetAsync(resid, 0, (size_t)max_iter * sizeof(double), st), "memset");
	const FlatTiles a = flat_tiles(f, m->carries.as<double>());
	AffOp op;
	op.nz_rows = f.nz_rows();
	op.w = w;
	op.base = base;
	op.d = d;
	op.tol = tol;
	op.E = (uint32_t)f.E;
	const uint32_t* off = f.off.as<uint32_t>();
	const int ctas = (int)tune_value(s->device, LG_TUNE_PR_CTAS_PER_SM);
	int sms = 148;
	if (ctas > 0) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->device);
	aff_empty_rows<<<grid_for(V, 256), 256, 0, st>>>(off, V, base, A, B, resid);
	s->launches++;
	int done = -1;          // iterations after which the residual fell below tol
	int issued = 0, chunk = 0, prev_first = 0, prev_n = 0;
	double r = 0.0;
	// waits for chunk c's residual copy and finds the first one below tol
	auto check = [&](int c, int first, int cnt) -> lg_status {
		LG_CUDA(cudaEventSynchronize(m->chunk_done[c & 1]), "adjoint step");
		const double* h = m->resid_host + (c & 1) * kChunk;
		for (int k = 0; k < cnt && done < 0; k++) {
			r = h[k];
			if (r < tol) done = first + k + 1;
		}
		return LG_OK;
	};
	while (issued < max_iter && done < 0) {
		const int n = std::min(kChunk, max_iter - issued);
		for (int j = 0; j < n; j++) {
			const int it = issued + j;
			op.x = (it & 1) ? B : A;
			op.y = (it & 1) ? A : B;
			op.resid = resid + it;
			op.prev = it > 0 ? resid + it - 1 : nullptr;
			if (f.ntiles > 0) {
				launch_flat_sweep(a, op, sms, ctas, st, aff_flat_step, aff_flat_loop<4>,
						aff_flat_loop<6>, aff_flat_loop<8>);
				s->launches++;
			}
			if (f.ntiles > 1) {
				aff_flat_fixup<<<flat_fixup_blocks(f.ntiles), kFixupThreads, 0, st>>>(a, op);
				s->launches++;
			}
			if (it == 0) {
				// A is read again by the third iteration: its rows without
				// edges take their constant value now
				aff_empty_rows<<<grid_for(V, 256), 256, 0, st>>>(off, V, base, nullptr, A,
						nullptr);
				s->launches++;
			}
		}
		LG_CUDA(cudaGetLastError(), "adjoint step");
		LG_CUDA(cudaMemcpyAsync(m->resid_host + (chunk & 1) * kChunk, resid + issued,
				n * sizeof(double), cudaMemcpyDeviceToHost, st), "d2h");
		LG_CUDA(cudaEventRecord(m->chunk_done[chunk & 1], st), "event");
		s->d2h_bytes += n * sizeof(double);
		// the previous chunk's residuals are read while this one runs
		if (chunk > 0) LG_TRY(check(chunk - 1, prev_first, prev_n));
		prev_first = issued;
		prev_n = n;
		issued += n;
		chunk++;
	}
	if (done < 0 && chunk > 0) LG_TRY(check(chunk - 1, prev_first, prev_n));
	if (done < 0) done = max_iter;
	*iters = done;
	*resid_out = r;
	*out = (done & 1) ? B : A;
	return LG_OK;
}

lg_status stage_in(lg_store* s, const double* src, uint64_t n, DevBuf& buf, const double** dev) {
	if (is_device_pointer(src)) { *dev = src; return LG_OK; }
	LG_TRY(buf.reserve(std::max<uint64_t>(n, 1) * 8));
	LG_CUDA(cudaMemcpyAsync(buf.p, src, n * 8, cudaMemcpyHostToDevice, s->stream), "h2d");
	s->h2d_bytes += n * 8;
	*dev = buf.as<double>();
	return LG_OK;
}

} // namespace

void lg_free_adjoint_maps(lg_adjoint_maps* m) { delete m; }

extern "C" lg_status lg_pagerank_fwd(lg_snapshot* sn, const double* weights,
		const double* teleport, double damping, double tol, int max_iter, double* x,
		lg_adjoint** tape, lg_fixed_point_result* result) {
	clear_error();
	if (tape) *tape = nullptr;
	if (!sn || !weights || !teleport || !x) return set_error(LG_EINVAL, "null argument");
	if (!(damping > 0 && damping < 1)) return set_error(LG_EINVAL, "damping must be in (0, 1)");
	if (!(tol > 0) || max_iter <= 0) return set_error(LG_EINVAL, "tol and max_iter must be positive");
	if (!sn->in.present) return set_error(LG_ESTATE, "needs the in-CSR (reverse edges)");
	lg_store* s = sn->store;
	LG_CUDA(cudaSetDevice(s->device), "cudaSetDevice");
	cudaStream_t st = s->stream;
	const uint64_t V = sn->V;
	LG_TRY(ensure_maps(sn));
	lg_adjoint_maps* m = sn->adj_maps;
	const uint64_t E = m->E;
	const double *w, *v;
	LG_TRY(stage_in(s, weights, E, m->stage_w, &w));
	LG_TRY(stage_in(s, teleport, V, m->stage_v, &v));
	LG_TRY(m->base.reserve(V * 8));
	LG_TRY(m->win.reserve(std::max<uint64_t>(E, 1) * 8));
	LG_TRY(m->xa.reserve(V * 8));
	LG_TRY(m->xb.reserve(V * 8));
	scale_vec<<<grid_for(V, 256), 256, 0, st>>>(v, 1.0 - damping, V, m->base.as<double>());
	gather_weights<<<grid_for(E, 256), 256, 0, st>>>(m->in_pos.as<uint32_t>(), E, w,
			m->win.as<double>());
	LG_CUDA(cudaMemcpyAsync(m->xa.p, v, V * 8, cudaMemcpyDeviceToDevice, st), "d2d");
	LG_CUDA(cudaGetLastError(), "pagerank fwd");
	s->launches += 2;
	int it = 0;
	double r = 0;
	double* res = nullptr;
	LG_TRY(fixed_point(sn, m->fin, m->win.as<double>(), m->base.as<double>(), damping, tol,
			max_iter, &it, &r, &res));
	if (tape) {
		lg_adjoint* t = new (std::nothrow) lg_adjoint();
		if (!t) return set_error(LG_ENOMEM, "host allocation");
		t->snap = sn;
		t->d = damping;
		t->tol = tol;
		t->max_iter = max_iter;
		lg_status rs = t->x.reserve(V * 8);
		if (!rs) rs = t->w.reserve(std::max<uint64_t>(E, 1) * 8);
		if (rs) { delete t; return rs; }
		cudaError_t ce = cudaMemcpyAsync(t->x.p, res, V * 8, cudaMemcpyDeviceToDevice, st);
		if (ce == cudaSuccess)
			ce = cudaMemcpyAsync(t->w.p, w, E * 8, cudaMemcpyDeviceToDevice, st);
		if (ce != cudaSuccess) { delete t; return cuda_status(ce, "d2d"); }
		*tape = t;
	}
	LG_TRY(copy_out(s, x, res, V * 8));
	LG_CUDA(cudaStreamSynchronize(st), "pagerank fwd");
	if (result) { result->iterations = it; result->residual = r; }
	return LG_OK;
}

extern "C" lg_status lg_pagerank_bwd(lg_adjoint* t, const double* dldx, double* dldw,
		double* dlde, lg_fixed_point_result* result) {
	clear_error();
	if (!t || !dldx) return set_error(LG_EINVAL, "null argument");
	lg_snapshot* sn = t->snap;
	lg_store* s = sn->store;
	LG_CUDA(cudaSetDevice(s->device), "cudaSetDevice");
	cudaStream_t st = s->stream;
	const uint64_t V = sn->V;
	lg_adjoint_maps* m = sn->adj_maps;
	const uint64_t E = m->E;
	DevBuf outw, oute;
	const double* g;
	LG_TRY(stage_in(s, dldx, V, m->stage_g, &g));
	LG_TRY(m->xa.reserve(V * 8));
	LG_TRY(m->xb.reserve(V * 8));
	LG_CUDA(cudaMemcpyAsync(m->xa.p, g, V * 8, cudaMemcpyDeviceToDevice, st), "d2d");
	int it = 0;
	double r = 0;
	double* lam = nullptr;
	LG_TRY(fixed_point(sn, m->fout, t->w.as<double>(), g, t->d, t->tol, t->max_iter, &it, &r,
			&lam));
	if (dldw) {
		const bool dev = is_device_pointer(dldw);
		double* o = dldw;
		if (!dev) { LG_TRY(outw.reserve(std::max<uint64_t>(E, 1) * 8)); o = outw.as<double>(); }
		edge_grad<<<grid_for(E, 256), 256, 0, st>>>(m->src.as<uint32_t>(),
				m->fout.ids.as<uint32_t>(), E, t->d, lam, t->x.as<double>(), o);
		s->launches++;
		if (!dev) LG_TRY(copy_out(s, dldw, o, E * 8));
	}
	if (dlde) {
		const bool dev = is_device_pointer(dlde);
		double* o = dlde;
		if (!dev) { LG_TRY(oute.reserve(V * 8)); o = oute.as<double>(); }
		scale_vec<<<grid_for(V, 256), 256, 0, st>>>(lam, 1.0 - t->d, V, o);
		s->launches++;
		if (!dev) LG_TRY(copy_out(s, dlde, o, V * 8));
	}
	LG_CUDA(cudaGetLastError(), "pagerank bwd");
	LG_CUDA(cudaStreamSynchronize(st), "pagerank bwd");
	if (result) { result->iterations = it; result->residual = r; }
	return LG_OK;
}

extern "C" lg_status lg_adjoint_free(lg_adjoint* t) {
	delete t;
	return LG_OK;
}
