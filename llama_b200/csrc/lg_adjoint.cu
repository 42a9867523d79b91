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
// out-adjacency order (the order lg_snapshot_adjacency(dir 0) returns).  A
// per-snapshot map, built on first use, sends every live slot of the out-
// and in-CSR to that position; each call gathers the weights into slot
// order so both sweeps read them contiguously.
//
// Both sweeps are the same kernel: y[v] = base[v] + d * sum over v's slots
// of wslot[k] * x[nbr(k)], over balanced ranges of the slot space, with
// short vertices summed by one lane and long ones by the warp, and
// straddling vertices fixed up in range order (as in lg_pagerank.cu).
#include "lg_device.cuh"
#include "lg_expand.cuh"

#include <cmath>

namespace lg {

constexpr uint32_t kAdjRange = 2048;
constexpr int kAdjThreads = 256;
constexpr uint32_t kNoPos = 0xffffffffu;

struct AffArgs {
	SnapCsr g;
	const uint32_t* pos;      // V + 1 slot prefix of this direction
	uint32_t total, nranges;
	const double* wslot;      // weight per virtual slot (0 for deleted slots)
	const double* x;
	const double* base;
	double d;
	double* y;
	double* carry_first;
	double* carry_last;
	double* resid;            // sum |y - x|
};

__device__ __forceinline__ void aff_finish(const AffArgs& a, uint32_t v, double s,
		double* r) {
	const double y = __dadd_rn(__ldg(a.base + v), __dmul_rn(a.d, s));
	a.y[v] = y;
	*r += fabs(y - __ldg(a.x + v));
}

// sum over n slots starting at virtual slot k0 (= off slots into the
// vertex's chain starting at fragment f); one lane or the whole warp
template <bool kWarp>
__device__ __forceinline__ double aff_sum(const AffArgs& a, uint32_t f, uint32_t off,
		uint32_t n, uint32_t k0) {
	const uint32_t lane = kWarp ? (threadIdx.x & 31u) : 0u;
	const uint32_t stride = kWarp ? 32u : 1u;
	const LevelTab* lt = a.g.lt;
	uint2 fr = a.g.frags[f];
	while (off >= frag_len(fr)) { off -= frag_len(fr); fr = a.g.frags[++f]; }
	double s = 0.0;
	uint32_t done = 0;
	while (done < n) {
		const uint32_t lv = frag_level(fr);
		const uint32_t base = fr.x + off;
		const uint32_t m = min(frag_len(fr) - off, n - done);
		const uint32_t* ids = lt->ids[lv] + base;
		const double* wk = a.wslot + k0 + done;
		for (uint32_t i0 = 0; i0 < m; i0 += stride * 4) {
			uint32_t id[4];
			double wv[4];
#pragma unroll
			for (int u = 0; u < 4; u++) {
				const uint32_t i = i0 + u * stride + lane;
				wv[u] = 0.0;
				id[u] = 0;
				if (i < m) { wv[u] = __ldg(wk + i); id[u] = __ldg(ids + i); }
			}
#pragma unroll
			for (int u = 0; u < 4; u++)
				if (wv[u] != 0.0) s += wv[u] * __ldg(a.x + id[u]);
		}
		done += m;
		off = 0;
		if (done < n) fr = a.g.frags[++f];
	}
	if (kWarp)
		for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
	return s;
}

__global__ void __launch_bounds__(kAdjThreads)
aff_step(AffArgs a) {
	const uint32_t lane = threadIdx.x & 31u;
	const uint64_t r64 = (uint64_t)blockIdx.x * (kAdjThreads / 32) + (threadIdx.x >> 5);
	if (r64 >= a.nranges) return;
	const uint32_t r = (uint32_t)r64;
	const bool last_range = r == a.nranges - 1;
	const uint32_t ra = r * kAdjRange;
	const uint32_t rb = last_range ? a.total : min(a.total, ra + kAdjRange);
	uint32_t e_begin, e_end;
	range_entries(a.pos, (uint32_t)a.g.V, ra, rb, last_range, &e_begin, &e_end);
	double res = 0.0;
	for (uint32_t ew = e_begin; ew < e_end; ew += 32) {
		const Window w = load_window(a.g, nullptr, a.pos, ew, e_end, ra, rb);
		const uint32_t span = w.s1 - w.s0;
		const bool longe = w.valid && span >= 32;
		double s = 0.0;
		if (w.valid && !longe && span > 0)
			s = aff_sum<false>(a, w.f0, w.s0 - w.start, span, w.s0);
		for (unsigned m = __ballot_sync(0xffffffffu, longe); m; m &= m - 1) {
			const int t = __ffs(m) - 1;
			const double ws = aff_sum<true>(a, __shfl_sync(0xffffffffu, w.f0, t),
					__shfl_sync(0xffffffffu, w.s0 - w.start, t),
					__shfl_sync(0xffffffffu, span, t), __shfl_sync(0xffffffffu, w.s0, t));
			if ((int)lane == t) s = ws;
		}
		if (w.valid) {
			const uint32_t end = __ldg(a.pos + w.e + 1);
			if (w.start < ra) a.carry_first[r] = s;
			else if (end > rb) a.carry_last[r] = s;
			else aff_finish(a, w.v, s, &res);
		}
	}
	for (int o = 16; o > 0; o >>= 1) res += __shfl_down_sync(0xffffffffu, res, o);
	if (lane == 0 && res != 0.0) atomicAdd(a.resid, res);
}

__global__ void aff_fixup(AffArgs a) {
	const uint64_t q = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x + 1;
	double res = 0.0;
	if (q < a.nranges) {
		const uint32_t s = (uint32_t)q * kAdjRange;
		uint32_t lo = 0, hi = (uint32_t)a.g.V;
		while (lo < hi) {
			const uint32_t mid = (lo + hi + 1) >> 1;
			if (__ldg(a.pos + mid) <= s) lo = mid; else hi = mid - 1;
		}
		const uint32_t e = lo;
		if (e < a.g.V) {
			const uint32_t start = __ldg(a.pos + e), end = __ldg(a.pos + e + 1);
			if (start < s && start >= s - kAdjRange && end > s) {
				const uint32_t r2 = (end - 1) / kAdjRange;
				double t = __ldcg(a.carry_last + (q - 1));
				for (uint32_t x = (uint32_t)q; x <= r2; x++) t += __ldcg(a.carry_first + x);
				aff_finish(a, e, t, &res);
			}
		}
	}
	if (res != 0.0) atomicAdd(a.resid, res);
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

__global__ void u32_to_u64_scan_input(const uint32_t* deg, uint64_t V, uint32_t* out) {
	const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i < V) out[i] = deg[i];
}

__global__ void widen_prefix(const uint32_t* p32, uint64_t n, uint64_t* p64) {
	const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i <= n) p64[i] = p32[i];
}

} // namespace lg

using namespace lg;

struct lg_adjoint_maps {
	DevBuf out_pos, in_pos, src, dst, adj_off;
	uint64_t E = 0;
};

struct lg_adjoint {
	lg_snapshot* snap = nullptr;
	double d = 0.85, tol = 1e-12;
	int max_iter = 0;
	DevBuf x, w_out;   // converged scores; weights in out-slot order
};

namespace {

lg_status ensure_maps(lg_snapshot* sn) {
	if (sn->adj_maps) return LG_OK;
	lg_store* s = sn->store;
	cudaStream_t st = s->stream;
	const uint64_t V = sn->V;
	lg_adjoint_maps* m = new (std::nothrow) lg_adjoint_maps();
	if (!m) return set_error(LG_ENOMEM, "host allocation");
	const uint64_t E = sn->out.n_edges;
	if (E >= 0xffffffffull) { delete m; return set_error(LG_ENOTSUP, "more than 2^32-1 edges"); }
	m->E = E;
	lg_status r = LG_OK;
	DevBuf tmp, p32, scan_tmp, badb;
	if (!r) r = m->out_pos.reserve(std::max<uint64_t>(sn->out.n_frag_slots, 1) * 4);
	if (!r) r = m->in_pos.reserve(std::max<uint64_t>(sn->in.n_frag_slots, 1) * 4);
	if (!r) r = m->src.reserve(std::max<uint64_t>(E, 1) * 4);
	if (!r) r = m->dst.reserve(std::max<uint64_t>(E, 1) * 4);
	if (!r) r = m->adj_off.reserve((V + 1) * 8);
	if (!r) r = p32.reserve((V + 1) * 4);
	if (!r) r = badb.reserve(4);
	uint64_t tot = 0;
	if (!r) r = exclusive_scan_u32(sn->out.deg.as<uint32_t>(), p32.as<uint32_t>(), V, scan_tmp,
			st, &tot);
	if (r) { delete m; return r; }
	cudaMemsetAsync(badb.p, 0, 4, st);
	widen_prefix<<<grid_for(V + 1, 256), 256, 0, st>>>(p32.as<uint32_t>(), V,
			m->adj_off.as<uint64_t>());
	const SnapCsr out = sn->view(0), in = sn->view(1);
	adj_out_map<<<grid_for(V, 128), 128, 0, st>>>(out, sn->out.slot_off.as<uint32_t>(),
			m->adj_off.as<uint64_t>(), m->out_pos.as<uint32_t>(), m->src.as<uint32_t>(),
			m->dst.as<uint32_t>(), badb.as<uint32_t>());
	adj_in_map<<<grid_for(V, 128), 128, 0, st>>>(in, sn->in.slot_off.as<uint32_t>(), out,
			sn->out.slot_off.as<uint32_t>(), m->out_pos.as<uint32_t>(),
			m->in_pos.as<uint32_t>(), badb.as<uint32_t>());
	s->launches += 6;
	uint32_t bad = 0;
	cudaError_t ce = cudaGetLastError();
	if (ce == cudaSuccess) ce = cudaMemcpyAsync(&bad, badb.p, 4, cudaMemcpyDeviceToHost, st);
	if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
	if (ce != cudaSuccess) { delete m; return cuda_status(ce, "adjoint maps"); }
	if (bad || tot != E) {
		delete m;
		return set_error(LG_EINVAL, "out- and in-CSR of the snapshot disagree, or a "
				"fragment is not sorted by neighbour id");
	}
	sn->adj_maps = m;
	return LG_OK;
}

// Iterate y = base + d * (weighted pull of x) over direction `dir` until
// sum |y - x| < tol; x holds the start on entry and the result on exit.
lg_status fixed_point(lg_snapshot* sn, int dir, const double* wslot, const double* base,
		double d, double tol, int max_iter, DevBuf& x, DevBuf& y, int* iters,
		double* resid_out) {
	lg_store* s = sn->store;
	cudaStream_t st = s->stream;
	const SnapDir& sd = dir == 0 ? sn->out : sn->in;
	AffArgs a;
	a.g = sn->view(dir);
	a.pos = sd.slot_off.as<uint32_t>();
	a.total = (uint32_t)sd.n_frag_slots;
	a.nranges = (uint32_t)std::max<uint64_t>(1, (a.total + kAdjRange - 1) / kAdjRange);
	a.wslot = wslot;
	a.base = base;
	a.d = d;
	DevBuf carry, rb;
	LG_TRY(carry.reserve(2ull * a.nranges * 8));
	LG_TRY(rb.reserve(8));
	a.carry_first = carry.as<double>();
	a.carry_last = a.carry_first + a.nranges;
	a.resid = rb.as<double>();
	double* cur = x.as<double>();
	double* nxt = y.as<double>();
	double r = 0.0;
	int it = 0;
	while (it < max_iter) {
		a.x = cur;
		a.y = nxt;
		LG_CUDA(cudaMemsetAsync(rb.p, 0, 8, st), "memset");
		aff_step<<<grid_for(a.nranges, kAdjThreads / 32), kAdjThreads, 0, st>>>(a);
		if (a.nranges > 1) aff_fixup<<<grid_for(a.nranges, 256), 256, 0, st>>>(a);
		LG_CUDA(cudaGetLastError(), "adjoint step");
		s->launches += a.nranges > 1 ? 2 : 1;
		LG_CUDA(cudaMemcpyAsync(&r, rb.p, 8, cudaMemcpyDeviceToHost, st), "d2h");
		LG_CUDA(cudaStreamSynchronize(st), "adjoint step");
		s->d2h_bytes += 8;
		std::swap(cur, nxt);
		it++;
		if (r < tol) break;
	}
	if (cur != x.as<double>())
		LG_CUDA(cudaMemcpyAsync(x.p, cur, sn->V * 8, cudaMemcpyDeviceToDevice, st), "d2d");
	*iters = it;
	*resid_out = r;
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
	DevBuf wb, vb, base, win, xa, xb;
	const double *w, *v;
	LG_TRY(stage_in(s, weights, m->E, wb, &w));
	LG_TRY(stage_in(s, teleport, V, vb, &v));
	LG_TRY(base.reserve(V * 8));
	LG_TRY(win.reserve(std::max<uint64_t>(sn->in.n_frag_slots, 1) * 8));
	LG_TRY(xa.reserve(V * 8));
	LG_TRY(xb.reserve(V * 8));
	scale_vec<<<grid_for(V, 256), 256, 0, st>>>(v, 1.0 - damping, V, base.as<double>());
	gather_weights<<<grid_for(sn->in.n_frag_slots, 256), 256, 0, st>>>(
			m->in_pos.as<uint32_t>(), sn->in.n_frag_slots, w, win.as<double>());
	LG_CUDA(cudaMemcpyAsync(xa.p, v, V * 8, cudaMemcpyDeviceToDevice, st), "d2d");
	s->launches += 2;
	int it = 0;
	double r = 0;
	LG_TRY(fixed_point(sn, 1, win.as<double>(), base.as<double>(), damping, tol, max_iter,
			xa, xb, &it, &r));
	LG_TRY(copy_out(s, x, xa.p, V * 8));
	if (tape) {
		lg_adjoint* t = new (std::nothrow) lg_adjoint();
		if (!t) return set_error(LG_ENOMEM, "host allocation");
		t->snap = sn;
		t->d = damping;
		t->tol = tol;
		t->max_iter = max_iter;
		lg_status rs = t->x.reserve(V * 8);
		if (!rs) rs = t->w_out.reserve(std::max<uint64_t>(sn->out.n_frag_slots, 1) * 8);
		if (rs) { delete t; return rs; }
		LG_CUDA(cudaMemcpyAsync(t->x.p, xa.p, V * 8, cudaMemcpyDeviceToDevice, st), "d2d");
		gather_weights<<<grid_for(sn->out.n_frag_slots, 256), 256, 0, st>>>(
				m->out_pos.as<uint32_t>(), sn->out.n_frag_slots, w, t->w_out.as<double>());
		s->launches++;
		*tape = t;
	}
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
	DevBuf gb, la, lb2, outw, oute;
	const double* g;
	LG_TRY(stage_in(s, dldx, V, gb, &g));
	LG_TRY(la.reserve(V * 8));
	LG_TRY(lb2.reserve(V * 8));
	LG_CUDA(cudaMemcpyAsync(la.p, g, V * 8, cudaMemcpyDeviceToDevice, st), "d2d");
	int it = 0;
	double r = 0;
	LG_TRY(fixed_point(sn, 0, t->w_out.as<double>(), g, t->d, t->tol, t->max_iter, la, lb2,
			&it, &r));
	if (dldw) {
		const bool dev = is_device_pointer(dldw);
		double* o = dldw;
		if (!dev) { LG_TRY(outw.reserve(std::max<uint64_t>(m->E, 1) * 8)); o = outw.as<double>(); }
		edge_grad<<<grid_for(m->E, 256), 256, 0, st>>>(m->src.as<uint32_t>(),
				m->dst.as<uint32_t>(), m->E, t->d, la.as<double>(), t->x.as<double>(), o);
		s->launches++;
		if (!dev) LG_TRY(copy_out(s, dldw, o, m->E * 8));
	}
	if (dlde) {
		const bool dev = is_device_pointer(dlde);
		double* o = dlde;
		if (!dev) { LG_TRY(oute.reserve(V * 8)); o = oute.as<double>(); }
		scale_vec<<<grid_for(V, 256), 256, 0, st>>>(la.as<double>(), 1.0 - t->d, V, o);
		s->launches++;
		if (!dev) LG_TRY(copy_out(s, dlde, o, V * 8));
	}
	LG_CUDA(cudaStreamSynchronize(st), "pagerank bwd");
	if (result) { result->iterations = it; result->residual = r; }
	return LG_OK;
}

extern "C" lg_status lg_adjoint_free(lg_adjoint* t) {
	delete t;
	return LG_OK;
}
