// lg_bc.cu - Brandes betweenness centrality from explicit sources, FP64.
//
// Reference: ll_b_bc_random (benchmark/benchmarks/bc_random.h:55-193) over
// ll_bfs_template: per source s, sigma is pushed along down edges
// (level[w] == level[v] + 1, is_down_edge, ll_bfs_template.h:337-351) and
// the reverse sweep, deepest level first, sets
//   delta[v] = sum over down edges v->w of sigma[v] / sigma[w] * (1 + delta[w])
// and BC[v] += delta[v] for v != s (bc_random.h:73-111).  The reference
// accumulates in FP32 and picks sources with rand(); here sources are given
// and everything is FP64.  Sums go through FP64 atomics, so results agree
// with an exact evaluation to ~1e-15 relative, not bit for bit.
//
// lg_bc (plain): one source at a time.  The forward sweep is a top-down BFS
// over balanced frontier ranges that also adds sigma[v] into sigma[w] for
// every down edge; the backward sweep walks each level's out-edges.
//
// lg_bc_batched: 64 sources per pass.  Per vertex the pass keeps a 64-byte
// row of depths, a 512-byte row of sigma and one of delta.  Edges are spread
// over balanced ranges as in the plain kernels, but each edge of a chunk is
// then handled by the whole warp with lane j serving sources j and j + 32, so
// the edge's id is loaded once for 64 traversals and the per-source state is
// read as coalesced rows.
#include "lg_device.cuh"
#include "lg_expand.cuh"

namespace lg {

constexpr int32_t kBcUnreached = LG_UNREACHED;
constexpr uint32_t kBcRange = 1024;
constexpr int kBcThreads = 256;
constexpr int kLanes = 64;                 // sources per batch
constexpr uint8_t kNoDepth = 0xff;

__device__ __forceinline__ void bc_push(bool take, uint32_t item, uint32_t* list,
		unsigned long long* len) {
	const unsigned m = __ballot_sync(0xffffffffu, take);
	if (!m) return;
	const uint32_t lane = threadIdx.x & 31u;
	const int leader = __ffs(m) - 1;
	unsigned long long base = 0;
	if ((int)lane == leader) base = atomicAdd(len, (unsigned long long)__popc(m));
	base = __shfl_sync(0xffffffffu, base, leader);
	if (take) list[base + __popc(m & ((1u << lane) - 1u))] = item;
}

// ---------------------------------------------------------------------------
// Plain: one source
// ---------------------------------------------------------------------------

__global__ void bc_source_init(int32_t* level, double* sigma, double* delta,
		uint64_t V, uint32_t s, uint32_t* order) {
	const uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (v < V) {
		level[v] = (v == s) ? 0 : kBcUnreached;
		sigma[v] = (v == s) ? 1.0 : 0.0;
		delta[v] = 0.0;
	}
	if (v == 0) order[0] = s;
}

__global__ void __launch_bounds__(kBcThreads)
bc_forward(SnapCsr out, const uint32_t* fr, const uint32_t* pos, uint32_t n,
		uint32_t total, uint32_t nranges, int32_t* level, double* sigma, int32_t k,
		uint32_t* next, unsigned long long* ctr) {
	const uint64_t r = (uint64_t)blockIdx.x * (kBcThreads / 32) + (threadIdx.x >> 5);
	if (r >= nranges) return;
	range_for_each(out, fr, pos, n, total, nranges, kBcRange, (uint32_t)r,
		[&](bool act, uint32_t own, uint32_t v, uint32_t w, uint32_t, uint32_t) {
			bool won = false, down = false;
			if (act) {
				int32_t lw = __ldcg(level + w);
				if (lw == kBcUnreached) {
					won = atomicCAS(level + w, kBcUnreached, k + 1) == kBcUnreached;
					lw = k + 1;   // set by us or by a concurrent parent
				}
				down = lw == k + 1;
			}
			if (down) atomicAdd(sigma + w, __ldcg(sigma + v));
			bc_push(won, w, next, ctr);
		});
}

__global__ void __launch_bounds__(kBcThreads)
bc_backward(SnapCsr out, const uint32_t* fr, const uint32_t* pos, uint32_t n,
		uint32_t total, uint32_t nranges, const int32_t* level, const double* sigma,
		double* delta, int32_t k) {
	const uint64_t r = (uint64_t)blockIdx.x * (kBcThreads / 32) + (threadIdx.x >> 5);
	if (r >= nranges) return;
	range_for_each(out, fr, pos, n, total, nranges, kBcRange, (uint32_t)r,
		[&](bool act, uint32_t own, uint32_t v, uint32_t w, uint32_t, uint32_t) {
			double c = 0.0;
			if (act && __ldcg(level + w) == k + 1)
				c = __ldcg(sigma + v) / __ldcg(sigma + w) * (1.0 + __ldcg(delta + w));
			bool tail;
			const double sum = warp_segsum(c, own, &tail);
			if (tail && sum != 0.0) atomicAdd(delta + v, sum);
		});
}

__global__ void bc_accumulate(const uint32_t* lvl, uint32_t n, const double* delta,
		double* bc) {
	const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n) { const uint32_t v = lvl[i]; bc[v] += delta[v]; }
}

// ---------------------------------------------------------------------------
// Batched: 64 sources
// ---------------------------------------------------------------------------

// depth rows: kLanes bytes per vertex; sigma / delta rows: kLanes doubles.
__global__ void bc64_init(uint8_t* depth, uint64_t V) {
	const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i < V * (kLanes / 16)) ((uint4*)depth)[i] = make_uint4(~0u, ~0u, ~0u, ~0u);
}

__global__ void bc64_sources(const uint32_t* src, int nb, uint8_t* depth, double* sigma,
		uint32_t* stamp, uint32_t* list, unsigned long long* ctr) {
	// one thread: sources may repeat, each keeps its own lane
	if (blockIdx.x != 0 || threadIdx.x != 0) return;
	unsigned long long n = 0;
	for (int j = 0; j < nb; j++) {
		const uint32_t s = src[j];
		depth[(uint64_t)s * kLanes + j] = 0;
		sigma[(uint64_t)s * kLanes + j] = 1.0;
		if (stamp[s] != 1u) { stamp[s] = 1u; list[n++] = s; }
	}
	*ctr = n;
}

__global__ void __launch_bounds__(kBcThreads)
bc64_forward(SnapCsr out, const uint32_t* fr, const uint32_t* pos, uint32_t n,
		uint32_t total, uint32_t nranges, uint8_t* depth, double* sigma, uint32_t k,
		uint32_t* stamp, uint32_t* next, unsigned long long* ctr) {
	const uint32_t lane = threadIdx.x & 31u;
	const uint64_t r = (uint64_t)blockIdx.x * (kBcThreads / 32) + (threadIdx.x >> 5);
	if (r >= nranges) return;
	range_for_each(out, fr, pos, n, total, nranges, kBcRange, (uint32_t)r,
		[&](bool act, uint32_t own, uint32_t v, uint32_t w, uint32_t, uint32_t) {
			unsigned todo = __ballot_sync(0xffffffffu, act);
			while (todo) {
				const int t = __ffs(todo) - 1;
				todo &= todo - 1;
				const uint32_t tv = __shfl_sync(0xffffffffu, v, t);
				const uint32_t tw = __shfl_sync(0xffffffffu, w, t);
				const uint8_t* dv = depth + (uint64_t)tv * kLanes;
				uint8_t* dw = depth + (uint64_t)tw * kLanes;
				bool fresh = false;
#pragma unroll
				for (int h = 0; h < 2; h++) {
					const uint32_t j = lane + 32 * h;
					if (__ldcg(dv + j) == (uint8_t)k) {
						uint8_t d = __ldcg(dw + j);
						if (d == kNoDepth) { dw[j] = (uint8_t)(k + 1); d = (uint8_t)(k + 1); fresh = true; }
						if (d == (uint8_t)(k + 1))
							atomicAdd(sigma + (uint64_t)tw * kLanes + j,
									__ldcg(sigma + (uint64_t)tv * kLanes + j));
					}
				}
				if (__any_sync(0xffffffffu, fresh) && lane == 0
						&& atomicExch(stamp + tw, k + 2) != k + 2) {
					const unsigned long long p = atomicAdd(ctr, 1ull);
					next[p] = tw;
				}
			}
		});
}

__global__ void __launch_bounds__(kBcThreads)
bc64_backward(SnapCsr out, const uint32_t* fr, const uint32_t* pos, uint32_t n,
		uint32_t total, uint32_t nranges, const uint8_t* depth, const double* sigma,
		double* delta, uint32_t k) {
	const uint32_t lane = threadIdx.x & 31u;
	const uint64_t r = (uint64_t)blockIdx.x * (kBcThreads / 32) + (threadIdx.x >> 5);
	if (r >= nranges) return;
	uint32_t cur = 0xffffffffu;
	double acc0 = 0.0, acc1 = 0.0;
	range_for_each(out, fr, pos, n, total, nranges, kBcRange, (uint32_t)r,
		[&](bool act, uint32_t own, uint32_t v, uint32_t w, uint32_t, uint32_t) {
			unsigned todo = __ballot_sync(0xffffffffu, act);
			while (todo) {
				const int t = __ffs(todo) - 1;
				todo &= todo - 1;
				const uint32_t tv = __shfl_sync(0xffffffffu, v, t);
				const uint32_t tw = __shfl_sync(0xffffffffu, w, t);
				if (tv != cur) {
					if (cur != 0xffffffffu) {
						if (acc0 != 0.0) atomicAdd(delta + (uint64_t)cur * kLanes + lane, acc0);
						if (acc1 != 0.0) atomicAdd(delta + (uint64_t)cur * kLanes + lane + 32, acc1);
					}
					cur = tv;
					acc0 = acc1 = 0.0;
				}
				const uint8_t* dv = depth + (uint64_t)tv * kLanes;
				const uint8_t* dw = depth + (uint64_t)tw * kLanes;
#pragma unroll
				for (int h = 0; h < 2; h++) {
					const uint32_t j = lane + 32 * h;
					if (__ldg(dv + j) == (uint8_t)k && __ldg(dw + j) == (uint8_t)(k + 1)) {
						const double c = __ldg(sigma + (uint64_t)tv * kLanes + j)
							/ __ldg(sigma + (uint64_t)tw * kLanes + j)
							* (1.0 + __ldcg(delta + (uint64_t)tw * kLanes + j));
						if (h == 0) acc0 += c; else acc1 += c;
					}
				}
			}
		});
	if (cur != 0xffffffffu) {
		if (acc0 != 0.0) atomicAdd(delta + (uint64_t)cur * kLanes + lane, acc0);
		if (acc1 != 0.0) atomicAdd(delta + (uint64_t)cur * kLanes + lane + 32, acc1);
	}
}

// bc[v] += sum of delta[v][j] over the sources j that have v at depth k
// (v != source j); one warp per vertex of the level.
__global__ void bc64_accumulate(const uint32_t* lvl, uint32_t n, const uint8_t* depth,
		const double* delta, const uint32_t* src, int nb, uint32_t k, double* bc) {
	const uint32_t lane = threadIdx.x & 31u;
	const uint64_t i = (uint64_t)blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
	if (i >= n) return;
	const uint32_t v = lvl[i];
	double s = 0.0;
	for (int h = 0; h < 2; h++) {
		const uint32_t j = lane + 32 * h;
		if ((int)j < nb && depth[(uint64_t)v * kLanes + j] == (uint8_t)k && src[j] != v)
			s += delta[(uint64_t)v * kLanes + j];
	}
	for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
	if (lane == 0) bc[v] += s;
}

__global__ void clear_stamps(uint32_t* stamp, const uint32_t* list, uint64_t n) {
	const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n) stamp[list[i]] = 0;
}

} // namespace lg

using namespace lg;

namespace {

lg_status list_offsets(lg_store* s, const SnapCsr& g, const uint32_t* list, uint32_t n,
		DevBuf& cnt, DevBuf& pos, DevBuf& scan_tmp, uint64_t* total) {
	list_slots<<<grid_for(n, 256), 256, 0, s->stream>>>(g, list, n, cnt.as<uint32_t>());
	s->launches += 4;
	s->d2h_bytes += 8;
	return exclusive_scan_u32(cnt.as<uint32_t>(), pos.as<uint32_t>(), n, scan_tmp,
			s->stream, total);
}

lg_status read_u64(lg_store* s, const unsigned long long* d, uint64_t* h) {
	unsigned long long x = 0;
	LG_CUDA(cudaMemcpyAsync(&x, d, 8, cudaMemcpyDeviceToHost, s->stream), "d2h");
	LG_CUDA(cudaStreamSynchronize(s->stream), "bc");
	s->d2h_bytes += 8;
	*h = x;
	return LG_OK;
}

lg_status check_sources(lg_snapshot* sn, const int64_t* sources, int n) {
	if (!sn || (!sources && n > 0)) return set_error(LG_EINVAL, "null argument");
	if (n < 0) return set_error(LG_EINVAL, "negative source count");
	for (int i = 0; i < n; i++)
		if (sources[i] < 0 || (uint64_t)sources[i] >= sn->V)
			return set_error(LG_EINVAL, "source %lld out of range", (long long)sources[i]);
	return LG_OK;
}

} // namespace

extern "C" lg_status lg_bc(lg_snapshot* sn, const int64_t* sources, int n_sources,
		double* bc) {
	clear_error();
	if (!bc) return set_error(LG_EINVAL, "null output");
	LG_TRY(check_sources(sn, sources, n_sources));
	lg_store* s = sn->store;
	LG_CUDA(cudaSetDevice(s->device), "cudaSetDevice");
	cudaStream_t st = s->stream;
	const uint64_t V = sn->V;
	DevBuf level, sigma, delta, order, cnt, pos, scan_tmp, ctrb, bcb;
	LG_TRY(level.reserve(V * 4));
	LG_TRY(sigma.reserve(V * 8));
	LG_TRY(delta.reserve(V * 8));
	LG_TRY(order.reserve(V * 4));
	LG_TRY(cnt.reserve(V * 4));
	LG_TRY(pos.reserve((V + 1) * 4));
	LG_TRY(ctrb.reserve(8));
	const bool dev_out = is_device_pointer(bc);
	double* acc = bc;
	if (!dev_out) { LG_TRY(bcb.reserve(V * 8)); acc = bcb.as<double>(); }
	LG_CUDA(cudaMemsetAsync(acc, 0, V * 8, st), "memset");
	const SnapCsr out = sn->view(0);
	int32_t* lv = level.as<int32_t>();
	double* sg = sigma.as<double>();
	double* dl = delta.as<double>();
	uint32_t* ord = order.as<uint32_t>();
	unsigned long long* ctr = ctrb.as<unsigned long long>();
	std::vector<uint64_t> off;
	for (int i = 0; i < n_sources; i++) {
		const uint32_t src = (uint32_t)sources[i];
		bc_source_init<<<grid_for(V, 256), 256, 0, st>>>(lv, sg, dl, V, src, ord);
		s->launches++;
		off.assign({0, 1});
		for (int32_t k = 0;; k++) {
			const uint64_t b = off[k], n = off[k + 1] - off[k];
			if (n == 0) break;
			uint64_t total = 0;
			LG_TRY(list_offsets(s, out, ord + b, (uint32_t)n, cnt, pos, scan_tmp, &total));
			LG_CUDA(cudaMemsetAsync(ctr, 0, 8, st), "memset");
			const uint32_t nr = (uint32_t)((total + kBcRange - 1) / kBcRange);
			if (nr) {
				bc_forward<<<grid_for(nr, kBcThreads / 32), kBcThreads, 0, st>>>(out, ord + b,
						pos.as<uint32_t>(), (uint32_t)n, (uint32_t)total, nr, lv, sg, k,
						ord + off[k + 1], ctr);
				s->launches++;
			}
			LG_CUDA(cudaGetLastError(), "bc_forward");
			uint64_t produced = 0;
			LG_TRY(read_u64(s, ctr, &produced));
			off.push_back(off[k + 1] + produced);
		}
		// backward: levels D-1 .. 1 (the deepest level has no down edges)
		const int D = (int)off.size() - 2;           // levels 0..D-1 are non-empty
		for (int k = D - 2; k >= 1; k--) {
			const uint64_t b = off[k], n = off[k + 1] - off[k];
			uint64_t total = 0;
			LG_TRY(list_offsets(s, out, ord + b, (uint32_t)n, cnt, pos, scan_tmp, &total));
			const uint32_t nr = (uint32_t)((total + kBcRange - 1) / kBcRange);
			if (nr) {
				bc_backward<<<grid_for(nr, kBcThreads / 32), kBcThreads, 0, st>>>(out, ord + b,
						pos.as<uint32_t>(), (uint32_t)n, (uint32_t)total, nr, lv, sg, dl, k);
				s->launches++;
			}
			bc_accumulate<<<grid_for(n, 256), 256, 0, st>>>(ord + b, (uint32_t)n, dl, acc);
			s->launches++;
			LG_CUDA(cudaGetLastError(), "bc_backward");
		}
	}
	if (!dev_out) LG_TRY(copy_out(s, bc, acc, V * 8));
	LG_CUDA(cudaStreamSynchronize(st), "bc");
	return LG_OK;
}

extern "C" lg_status lg_bc_batched(lg_snapshot* sn, const int64_t* sources,
		int n_sources, double* bc) {
	clear_error();
	if (!bc) return set_error(LG_EINVAL, "null output");
	LG_TRY(check_sources(sn, sources, n_sources));
	lg_store* s = sn->store;
	LG_CUDA(cudaSetDevice(s->device), "cudaSetDevice");
	cudaStream_t st = s->stream;
	const uint64_t V = sn->V;
	DevBuf depth, sigma, delta, stamp, order, cnt, pos, scan_tmp, ctrb, srcb, bcb;
	LG_TRY(depth.reserve(V * kLanes));
	LG_TRY(sigma.reserve(V * kLanes * 8));
	LG_TRY(delta.reserve(V * kLanes * 8));
	LG_TRY(stamp.reserve(V * 4));
	LG_TRY(order.reserve(V * 4 * 8 + 64));   // concatenated level lists
	LG_TRY(cnt.reserve(V * 4));
	LG_TRY(pos.reserve((V + 1) * 4));
	LG_TRY(ctrb.reserve(8));
	LG_TRY(srcb.reserve(kLanes * 4));
	const bool dev_out = is_device_pointer(bc);
	double* acc = bc;
	if (!dev_out) { LG_TRY(bcb.reserve(V * 8)); acc = bcb.as<double>(); }
	LG_CUDA(cudaMemsetAsync(acc, 0, V * 8, st), "memset");
	LG_CUDA(cudaMemsetAsync(stamp.p, 0, V * 4, st), "memset");
	const SnapCsr out = sn->view(0);
	uint8_t* dp = depth.as<uint8_t>();
	double* sg = sigma.as<double>();
	double* dl = delta.as<double>();
	uint32_t* st_ = stamp.as<uint32_t>();
	uint32_t* ord = order.as<uint32_t>();
	const uint64_t ord_cap = V * 8 + 16;
	unsigned long long* ctr = ctrb.as<unsigned long long>();
	uint32_t* srcd = srcb.as<uint32_t>();
	std::vector<uint64_t> off;
	for (int b0 = 0; b0 < n_sources; b0 += kLanes) {
		const int nb = std::min(kLanes, n_sources - b0);
		uint32_t hs[kLanes];
		for (int j = 0; j < kLanes; j++) hs[j] = j < nb ? (uint32_t)sources[b0 + j] : 0xffffffffu;
		LG_CUDA(cudaMemcpyAsync(srcd, hs, sizeof(hs), cudaMemcpyHostToDevice, st), "h2d");
		s->h2d_bytes += sizeof(hs);
		bc64_init<<<grid_for(V * (kLanes / 16), 256), 256, 0, st>>>(dp, V);
		LG_CUDA(cudaMemsetAsync(sg, 0, V * kLanes * 8, st), "memset");
		LG_CUDA(cudaMemsetAsync(dl, 0, V * kLanes * 8, st), "memset");
		bc64_sources<<<1, 32, 0, st>>>(srcd, nb, dp, sg, st_, ord, ctr);
		s->launches += 2;
		uint64_t n0 = 0;
		LG_TRY(read_u64(s, ctr, &n0));
		off.assign({0, n0});
		for (uint32_t k = 0;; k++) {
			const uint64_t b = off[k], n = off[k + 1] - off[k];
			if (n == 0) break;
			if (k + 2 >= 0xff) return set_error(LG_ENOTSUP, "BFS deeper than 253 levels");
			if (off[k + 1] + V > ord_cap)
				return set_error(LG_ENOTSUP, "level lists exceed their buffer");
			uint64_t total = 0;
			LG_TRY(list_offsets(s, out, ord + b, (uint32_t)n, cnt, pos, scan_tmp, &total));
			LG_CUDA(cudaMemsetAsync(ctr, 0, 8, st), "memset");
			const uint32_t nr = (uint32_t)((total + kBcRange - 1) / kBcRange);
			if (nr) {
				bc64_forward<<<grid_for(nr, kBcThreads / 32), kBcThreads, 0, st>>>(out, ord + b,
						pos.as<uint32_t>(), (uint32_t)n, (uint32_t)total, nr, dp, sg, k, st_,
						ord + off[k + 1], ctr);
				s->launches++;
			}
			LG_CUDA(cudaGetLastError(), "bc64_forward");
			uint64_t produced = 0;
			LG_TRY(read_u64(s, ctr, &produced));
			off.push_back(off[k + 1] + produced);
		}
		// levels D-1 .. 1; level 0 holds only the sources, which BC excludes
		const int D = (int)off.size() - 2;
		for (int k = D - 1; k >= 1; k--) {
			const uint64_t b = off[k], n = off[k + 1] - off[k];
			uint64_t total = 0;
			LG_TRY(list_offsets(s, out, ord + b, (uint32_t)n, cnt, pos, scan_tmp, &total));
			const uint32_t nr = (uint32_t)((total + kBcRange - 1) / kBcRange);
			if (nr && k < D - 1) {
				bc64_backward<<<grid_for(nr, kBcThreads / 32), kBcThreads, 0, st>>>(out, ord + b,
						pos.as<uint32_t>(), (uint32_t)n, (uint32_t)total, nr, dp, sg, dl, k);
				s->launches++;
			}
			bc64_accumulate<<<grid_for(n, 8), 256, 0, st>>>(ord + b, (uint32_t)n, dp, dl,
					srcd, nb, k, acc);
			s->launches++;
			LG_CUDA(cudaGetLastError(), "bc64_backward");
		}
		// reset the stamps of every listed vertex for the next batch
		clear_stamps<<<grid_for(off.back(), 256), 256, 0, st>>>(st_, ord, off.back());
		s->launches++;
	}
	if (!dev_out) LG_TRY(copy_out(s, bc, acc, V * 8));
	LG_CUDA(cudaStreamSynchronize(st), "bc batched");
	return LG_OK;
}
