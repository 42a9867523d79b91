// lg_store.cu - device mirror of the LLAMA level stack: ingest of levels in
// the reference's layout, snapshot views (fragment walk + deletion bitset),
// degree and adjacency queries, and the error plumbing of the C ABI.
#include "lg_device.cuh"
#include "lg_flat.cuh"

#include <omp.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

namespace lg {

// ---------------------------------------------------------------------------
// Errors
// ---------------------------------------------------------------------------

static thread_local char t_err[512];

lg_status set_error(lg_status st, const char* fmt, ...) {
	va_list ap;
	va_start(ap, fmt);
	vsnprintf(t_err, sizeof(t_err), fmt, ap);
	va_end(ap);
	return st;
}

void clear_error() { t_err[0] = 0; }

lg_status cuda_status(cudaError_t e, const char* what) {
	if (e == cudaErrorMemoryAllocation)
		return set_error(LG_ENOMEM, "%s: %s", what, cudaGetErrorString(e));
	return set_error(LG_ECUDA, "%s: %s", what, cudaGetErrorString(e));
}

lg_status DevBuf::reserve(size_t n) {
	if (n <= bytes && p) return LG_OK;
	release();
	if (n == 0) n = 16;
	cudaError_t e = cudaMalloc(&p, n);
	if (e != cudaSuccess) {
		p = nullptr;
		(void)cudaGetLastError();
		return cuda_status(e, "cudaMalloc");
	}
	bytes = n;
	return LG_OK;
}

bool is_device_pointer(const void* ptr) {
	cudaPointerAttributes a;
	cudaError_t e = cudaPointerGetAttributes(&a, ptr);
	if (e != cudaSuccess) { (void)cudaGetLastError(); return false; }
	return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

static bool is_pinned_host(const void* ptr) {
	cudaPointerAttributes a;
	cudaError_t e = cudaPointerGetAttributes(&a, ptr);
	if (e != cudaSuccess) { (void)cudaGetLastError(); return false; }
	return a.type == cudaMemoryTypeHost;
}

// LG_OUTPUT_ASYNC: the result is copied into a staging slot on the store's
// stream (so the caller may reuse `src` at once) and from there to the host
// on copy_stream.  The slot is reused only after its previous copy ended.
static lg_status copy_out_async(lg_store* s, void* dst, const void* src, size_t bytes) {
	if (!s->copy_stream) {
		LG_CUDA(cudaStreamCreateWithFlags(&s->copy_stream, cudaStreamNonBlocking), "copy stream");
		for (int i = 0; i < 2; i++) {
			LG_CUDA(cudaEventCreateWithFlags(&s->stage_ready[i], cudaEventDisableTiming), "event");
			LG_CUDA(cudaEventCreateWithFlags(&s->stage_done[i], cudaEventDisableTiming), "event");
		}
	}
	const int i = s->stage_next;
	s->stage_next ^= 1;
	DevBuf& b = s->out_stage[i];
	if (bytes > b.bytes) {
		// the old buffer may still be read by the slot's previous copy
		LG_CUDA(cudaStreamSynchronize(s->copy_stream), "copy stream");
		LG_TRY(b.reserve(bytes));
	}
	LG_CUDA(cudaStreamWaitEvent(s->stream, s->stage_done[i], 0), "wait for slot");
	LG_CUDA(cudaMemcpyAsync(b.p, src, bytes, cudaMemcpyDeviceToDevice, s->stream), "stage result");
	LG_CUDA(cudaEventRecord(s->stage_ready[i], s->stream), "event");
	LG_CUDA(cudaStreamWaitEvent(s->copy_stream, s->stage_ready[i], 0), "wait for result");
	LG_CUDA(cudaMemcpyAsync(dst, b.p, bytes, cudaMemcpyDeviceToHost, s->copy_stream),
			"copy result");
	LG_CUDA(cudaEventRecord(s->stage_done[i], s->copy_stream), "event");
	s->d2h_bytes += bytes;
	return LG_OK;
}

lg_status host_words(lg_store* s, unsigned long long** words) {
	if (!s->host_words)
		LG_CUDA(cudaHostAlloc((void**)&s->host_words, kHostWords * sizeof(unsigned long long),
				cudaHostAllocDefault), "cudaHostAlloc");
	*words = s->host_words;
	return LG_OK;
}

lg_status read_words(lg_store* s, const unsigned long long* dev, int n, unsigned long long* out) {
	unsigned long long* hw = nullptr;
	LG_TRY(host_words(s, &hw));
	hw += 8;
	LG_CUDA(cudaMemcpyAsync(hw, dev, (size_t)n * sizeof(unsigned long long),
			cudaMemcpyDeviceToHost, s->stream), "d2h");
	LG_CUDA(cudaStreamSynchronize(s->stream), "d2h");
	for (int i = 0; i < n; i++) out[i] = hw[i];
	s->d2h_bytes += (uint64_t)n * sizeof(unsigned long long);
	return LG_OK;
}

lg_status copy_out(lg_store* s, void* dst, const void* src, size_t bytes) {
	if (bytes == 0) return LG_OK;
	if (s->output_mode == LG_OUTPUT_ASYNC && bytes >= LG_ASYNC_MIN_BYTES && is_pinned_host(dst))
		return copy_out_async(s, dst, src, bytes);
	if (!is_device_pointer(dst)) s->d2h_bytes += bytes;
	LG_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, s->stream), "copy result");
	return LG_OK;
}

DevLevel* take_level(lg_store* s, int dir) {
	DevLevel* d = s->level_spare[dir];
	s->level_spare[dir] = nullptr;
	if (!d) return new (std::nothrow) DevLevel();
	d->max_nodes = d->n_slots = d->n_fragment_slots = 0;
	return d;
}

lg_status append_dels(lg_store* s, DevCsr& csr, const uint2* add, size_t n,
		cudaMemcpyKind kind) {
	const size_t old_n = csr.n_dels_dev;
	const size_t need = (old_n + n) * sizeof(uint2);
	if (need > csr.dels.bytes) {
		// a larger list keeps the marks already on the device
		DevBuf nb;
		LG_TRY(nb.reserve(need + need / 2));
		if (old_n)
			LG_CUDA(cudaMemcpyAsync(nb.p, csr.dels.p, old_n * sizeof(uint2),
					cudaMemcpyDeviceToDevice, s->stream), "deletion list");
		// the old list may still be read by queued kernels
		LG_CUDA(cudaStreamSynchronize(s->stream), "deletion list");
		csr.dels.swap(nb);
	}
	if (n) {
		// (a pageable host source is copied before cudaMemcpyAsync returns)
		LG_CUDA(cudaMemcpyAsync(csr.dels.as<uint2>() + old_n, add, n * sizeof(uint2), kind,
				s->stream), "deletion list");
		if (kind == cudaMemcpyHostToDevice) s->h2d_bytes += n * sizeof(uint2);
	}
	csr.dels_mark.push_back(old_n);
	csr.n_dels_dev = old_n + n;
	return LG_OK;
}

// ---------------------------------------------------------------------------
// Exclusive scan (u32 -> u32): per-tile sums, a single-CTA scan of the tile
// sums, then per-tile scans with the carried offset.
// ---------------------------------------------------------------------------

constexpr int kScanThreads = 1024;
constexpr int kScanItems = 8;
constexpr uint64_t kScanTile = (uint64_t)kScanThreads * kScanItems;

__device__ __forceinline__ uint64_t block_excl_scan(uint64_t x, uint64_t* total) {
	__shared__ uint64_t warp_sums[32];
	const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
	uint64_t v = x;
#pragma unroll
	for (int o = 1; o < 32; o <<= 1) {
		uint64_t t = __shfl_up_sync(0xffffffffu, v, o);
		if (lane >= o) v += t;
	}
	if (lane == 31) warp_sums[wid] = v;
	__syncthreads();
	if (wid == 0) {
		int nw = blockDim.x >> 5;
		uint64_t s = lane < nw ? warp_sums[lane] : 0;
#pragma unroll
		for (int o = 1; o < 32; o <<= 1) {
			uint64_t t = __shfl_up_sync(0xffffffffu, s, o);
			if (lane >= o) s += t;
		}
		if (lane < nw) warp_sums[lane] = s;
	}
	__syncthreads();
	uint64_t before = wid > 0 ? warp_sums[wid - 1] : 0;
	*total = warp_sums[(blockDim.x >> 5) - 1];
	__syncthreads();
	return before + v - x;
}

__global__ void scan_tile_sums(const uint32_t* in, uint64_t n, uint64_t* sums) {
	uint64_t base = (uint64_t)blockIdx.x * kScanTile;
	uint64_t s = 0;
	for (int i = 0; i < kScanItems; i++) {
		uint64_t idx = base + (uint64_t)i * kScanThreads + threadIdx.x;
		if (idx < n) s += in[idx];
	}
	uint64_t tot;
	block_excl_scan(s, &tot);
	if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

__global__ void scan_sums_single(uint64_t* sums, uint64_t n, uint64_t* grand) {
	uint64_t carry = 0;
	for (uint64_t b = 0; b < n; b += kScanThreads) {
		uint64_t i = b + threadIdx.x;
		uint64_t x = i < n ? sums[i] : 0, tot;
		uint64_t ex = block_excl_scan(x, &tot);
		if (i < n) sums[i] = carry + ex;
		carry += tot;
	}
	if (threadIdx.x == 0) *grand = carry;
}

// A thread scans kScanItems consecutive values; with 16-byte aligned arrays
// it moves them as two 16-byte vectors each way.
__global__ void scan_tiles(const uint32_t* in, uint32_t* out, uint64_t n,
		const uint64_t* sums, const uint64_t* grand) {
	static_assert(kScanItems == 8, "two 16-byte vectors per thread");
	uint64_t base = (uint64_t)blockIdx.x * kScanTile
		+ (uint64_t)threadIdx.x * kScanItems;
	const bool vec = ((((uintptr_t)in) | ((uintptr_t)out)) & 15u) == 0 && base + kScanItems <= n;
	uint32_t vals[kScanItems];
	if (vec) {
		const uint4 a = __ldcs(reinterpret_cast<const uint4*>(in + base));
		const uint4 b = __ldcs(reinterpret_cast<const uint4*>(in + base + 4));
		vals[0] = a.x; vals[1] = a.y; vals[2] = a.z; vals[3] = a.w;
		vals[4] = b.x; vals[5] = b.y; vals[6] = b.z; vals[7] = b.w;
	} else {
#pragma unroll
		for (int i = 0; i < kScanItems; i++) {
			uint64_t idx = base + i;
			vals[i] = idx < n ? in[idx] : 0;
		}
	}
	uint64_t s = 0;
#pragma unroll
	for (int i = 0; i < kScanItems; i++) s += vals[i];
	uint64_t tot;
	uint64_t ex = block_excl_scan(s, &tot) + sums[blockIdx.x];
	uint32_t o[kScanItems];
#pragma unroll
	for (int i = 0; i < kScanItems; i++) {
		o[i] = (uint32_t)ex;
		ex += vals[i];
	}
	if (vec) {
		reinterpret_cast<uint4*>(out + base)[0] = make_uint4(o[0], o[1], o[2], o[3]);
		reinterpret_cast<uint4*>(out + base)[1] = make_uint4(o[4], o[5], o[6], o[7]);
	} else {
#pragma unroll
		for (int i = 0; i < kScanItems; i++) {
			uint64_t idx = base + i;
			if (idx < n) out[idx] = o[i];
		}
	}
	if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) out[n] = (uint32_t)*grand;
}

lg_status exclusive_scan_u32(const uint32_t* in, uint32_t* out, uint64_t n,
		DevBuf& tmp, cudaStream_t stream, uint64_t* total) {
	uint64_t tiles = (n + kScanTile - 1) / kScanTile;
	if (tiles == 0) tiles = 1;
	LG_TRY(tmp.reserve((tiles + 1) * sizeof(uint64_t)));
	uint64_t* sums = tmp.as<uint64_t>();
	scan_tile_sums<<<(unsigned)tiles, kScanThreads, 0, stream>>>(in, n, sums);
	scan_sums_single<<<1, kScanThreads, 0, stream>>>(sums, tiles, sums + tiles);
	scan_tiles<<<(unsigned)tiles, kScanThreads, 0, stream>>>(in, out, n, sums,
			sums + tiles);
	LG_CUDA(cudaGetLastError(), "scan launch");
	if (total) {
		// read through one pinned word per host thread (kept for the
		// thread's life): per-level loops read a total every step
		static thread_local uint64_t* pinned_total = nullptr;
		if (!pinned_total)
			LG_CUDA(cudaHostAlloc((void**)&pinned_total, sizeof(uint64_t),
					cudaHostAllocPortable), "cudaHostAlloc");
		LG_CUDA(cudaMemcpyAsync(pinned_total, sums + tiles, sizeof(uint64_t),
				cudaMemcpyDeviceToHost, stream), "scan total");
		LG_CUDA(cudaStreamSynchronize(stream), "scan total");
		const uint64_t t = *pinned_total;
		*total = t;
		if (t > 0xffffffffull)
			return set_error(LG_ENOTSUP, "more than 2^32-1 fragments in a snapshot");
	}
	return LG_OK;
}

// ---------------------------------------------------------------------------
// Ingest
// ---------------------------------------------------------------------------

static constexpr size_t kStageHalf = 64ull << 20;   // bytes per staging half

static lg_status ensure_staging(lg_store* s) {
	if (s->pinned) return LG_OK;
	LG_CUDA(cudaHostAlloc(&s->pinned, 2 * kStageHalf, cudaHostAllocDefault),
			"pinned staging");
	s->pinned_bytes = 2 * kStageHalf;
	for (int i = 0; i < 2; i++)
		LG_CUDA(cudaEventCreateWithFlags(&s->staged[i], cudaEventDisableTiming),
				"staging event");
	return LG_OK;
}

// Stream `bytes` to device memory `dst` through the pinned halves; `fill`
// writes bytes [off, off + n) of the source image into the staging buffer.
template <class Fill>
static lg_status staged_copy(lg_store* s, void* dst, size_t bytes, Fill&& fill) {
	LG_TRY(ensure_staging(s));
	size_t off = 0;
	int half = 0;
	while (off < bytes) {
		size_t n = std::min(kStageHalf, bytes - off);
		char* st = (char*)s->pinned + half * kStageHalf;
		LG_CUDA(cudaEventSynchronize(s->staged[half]), "staging wait");
		lg_status fs = fill(st, off, n);
		if (fs) return fs;
		LG_CUDA(cudaMemcpyAsync((char*)dst + off, st, n,
				cudaMemcpyHostToDevice, s->stream), "ingest copy");
		LG_CUDA(cudaEventRecord(s->staged[half], s->stream), "staging event");
		s->h2d_bytes += n;
		off += n;
		half ^= 1;
	}
	return LG_OK;
}

static inline const lg_vt_entry& vt_at(const lg_csr_level& c, uint64_t v) {
	if (c.vt) return c.vt[v];
	return c.vt_pages[v >> 9][v & 511];
}

static lg_status ingest_csr(lg_store* s, DevCsr& csr, int l,
		const lg_csr_level& c, const lg_deletion* dels, uint64_t n_dels,
		const char* name) {
	const uint64_t V = c.max_nodes;
	const uint64_t S = c.n_slots;
	if (V == 0 || V >= 0xffffffffull)
		return set_error(LG_EINVAL, "%s: max_nodes must be in [1, 2^32-1)", name);
	if (S >= 0xffffffffull)
		return set_error(LG_ENOTSUP, "%s: more than 2^32-1 slots in one level", name);
	if ((c.vt == nullptr) == (c.vt_pages == nullptr))
		return set_error(LG_EINVAL, "%s: exactly one of vt / vt_pages must be set", name);
	if (S > 0 && !c.slots)
		return set_error(LG_EINVAL, "%s: slots missing", name);

	// Validate the vertex table and mark the slots that belong to fragments
	// of this level.
	std::vector<uint8_t> mask(S, 0);
	int bad = 0;
	uint64_t frag_slots = 0;
	const auto& lv = csr.levels;
#pragma omp parallel for schedule(dynamic, 65536) reduction(|:bad) reduction(+:frag_slots)
	for (uint64_t v = 0; v < V; v++) {
		const lg_vt_entry& e = vt_at(c, v);
		if (e.adj_list_start == LG_NIL_EDGE || e.level_length == 0) continue;
		uint32_t el = LG_EDGE_LEVEL(e.adj_list_start);
		uint64_t ix = LG_EDGE_INDEX(e.adj_list_start);
		if (e.level_length > LG_MAX_FRAGMENT_LEN) { bad |= 4; continue; }
		if ((int)el > l) { bad |= 1; continue; }
		uint64_t lim = (int)el == l ? S : lv[el]->n_slots;
		if (ix + e.level_length > lim) { bad |= 2; continue; }
		if ((int)el == l) {
			for (uint64_t k = 0; k < e.level_length; k++) mask[ix + k] = 1;
			frag_slots += e.level_length;
		}
	}
	if (bad & 4) return set_error(LG_ENOTSUP, "%s: fragment longer than %u slots", name, LG_MAX_FRAGMENT_LEN);
	if (bad & 1) return set_error(LG_EINVAL, "%s: vertex table points to a future level", name);
	if (bad & 2) return set_error(LG_EINVAL, "%s: fragment exceeds its edge table", name);

	DevLevel* d = take_level(s, &csr == &s->out ? 0 : 1);
	if (!d) return set_error(LG_ENOMEM, "host allocation");
	d->max_nodes = V;
	d->n_slots = S;
	d->n_fragment_slots = frag_slots;
	if (!c.weights) d->w.release();
	lg_status st = d->vt.reserve((V + 1) * sizeof(lg_vt_entry));
	if (!st) st = d->ids.reserve(std::max<uint64_t>(S, 1) * sizeof(uint32_t));
	if (!st && c.weights) st = d->w.reserve(std::max<uint64_t>(S, 1) * sizeof(uint32_t));
	if (st) { delete d; return st; }

	// vertex table
	st = staged_copy(s, d->vt.p, (V + 1) * sizeof(lg_vt_entry),
		[&](char* dst, size_t off, size_t n) -> lg_status {
			uint64_t e0 = off / sizeof(lg_vt_entry), ne = n / sizeof(lg_vt_entry);
			lg_vt_entry* o = (lg_vt_entry*)dst;
#pragma omp parallel for schedule(static)
			for (uint64_t i = 0; i < ne; i++) o[i] = vt_at(c, e0 + i);
			return LG_OK;
		});
	// neighbour ids; slots already carrying a lowered max_visible_level
	// become deletion entries
	std::vector<std::vector<uint2>> found(omp_get_max_threads());
	int bad_id = 0;
	if (!st) st = staged_copy(s, d->ids.p, S * sizeof(uint32_t),
		[&](char* dst, size_t off, size_t n) -> lg_status {
			uint64_t i0 = off / 4, ni = n / 4;
			uint32_t* o = (uint32_t*)dst;
			int b = 0;
#pragma omp parallel reduction(|:b)
			{
				std::vector<uint2>& f = found[omp_get_thread_num()];
#pragma omp for schedule(static)
				for (uint64_t i = 0; i < ni; i++) {
					uint64_t k = i0 + i;
					if (!mask[k]) { o[i] = kNoId; continue; }
					uint64_t slot = c.slots[k];
					uint64_t pay = LG_SLOT_PAYLOAD(slot);
					if (pay >= V) { b |= 1; o[i] = kNoId; continue; }
					o[i] = (uint32_t)pay;
					uint32_t ml = LG_SLOT_MAX_LEVEL(slot);
					if (ml != LG_FRESH_MAX_LEVEL)
						f.push_back(make_uint2((uint32_t)k,
								((uint32_t)l << LG_BITS_LEVEL) | ml));
				}
			}
			bad_id |= b;
			return LG_OK;
		});
	if (!st && bad_id) st = set_error(LG_EINVAL, "%s: neighbour id >= max_nodes", name);
	if (!st && c.weights) st = staged_copy(s, d->w.p, S * sizeof(uint32_t),
		[&](char* dst, size_t off, size_t n) -> lg_status {
			std::memcpy(dst, (const char*)c.weights + off, n);
			return LG_OK;
		});
	if (st) {
		cudaStreamSynchronize(s->stream);
		delete d;
		return st;
	}
	// deletion marks in older levels
	std::vector<uint2> add;
	for (auto& f : found) add.insert(add.end(), f.begin(), f.end());
	for (uint64_t i = 0; i < n_dels; i++) {
		const lg_deletion& x = dels[i];
		uint32_t el = LG_EDGE_LEVEL(x.edge);
		uint64_t ix = LG_EDGE_INDEX(x.edge);
		if (x.edge < 0 || (int)el >= l || ix >= lv[el]->n_slots
				|| x.max_visible_level >= LG_FRESH_MAX_LEVEL) {
			cudaStreamSynchronize(s->stream);
			delete d;
			return set_error(LG_EINVAL, "%s: deletion %llu does not name an older slot",
					name, (unsigned long long)i);
		}
		add.push_back(make_uint2((uint32_t)ix, (el << LG_BITS_LEVEL) | x.max_visible_level));
	}
	csr.levels.push_back(d);
	return append_dels(s, csr, add.data(), add.size(), cudaMemcpyHostToDevice);
}

// ---------------------------------------------------------------------------
// Snapshot construction
// ---------------------------------------------------------------------------

struct VtTab {
	const lg_vt_entry* vt[LG_MAX_LEVELS];
	uint64_t max_nodes[LG_MAX_LEVELS];
};

// Fragment chain of v in snapshot L: iter_begin + iter_descend
// (llama/include/llama/ll_mlcsr_sp.h:1994-2134).  The continuation record read
// by iter_descend is the element VT[level-1][v] copied when `level` was built
// (ll_mlcsr_sp.h:1474-1497) and older levels never change afterwards, so the
// walk reads that element directly.
//
// With a minimum level minL (the sliding window), the chain ends at the first
// fragment of a level below minL, as iter_begin / iter_descend end it under
// LL_MIN_LEVEL (ll_mlcsr_sp.h:2021-2026, 2107-2110); vertex tables of levels
// below minL are never read.
template <bool kFill>
__global__ void walk_fragments(VtTab tab, int L, int minL, uint64_t V, uint32_t* count,
		uint32_t* deg, uint32_t* slots_per_vertex, const uint32_t* frag_off,
		uint2* frags) {
	uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (v >= V) return;
	lg_vt_entry e = tab.vt[L][v];
	if (!kFill) deg[v] = e.degree;
	uint32_t n = 0, slots = 0;
	uint32_t out = kFill ? frag_off[v] : 0;
	while (e.adj_list_start != LG_NIL_EDGE && e.level_length != 0) {
		uint32_t lv = LG_EDGE_LEVEL(e.adj_list_start);
		if ((int)lv < minL) break;
		uint32_t ix = (uint32_t)LG_EDGE_INDEX(e.adj_list_start);
		if (kFill) frags[out + n] = make_uint2(ix, (e.level_length << kLevelBits) | lv);
		n++;
		slots += e.level_length;
		if ((int)lv <= minL || v >= tab.max_nodes[lv - 1]) break;
		e = tab.vt[lv - 1][v];
	}
	if (!kFill) { count[v] = n; slots_per_vertex[v] = slots; }
}

__global__ void live_counts(SnapCsr g, uint32_t* out);

// Sets the bit of every slot deleted at or before L and counts them in *count.
// Slots of levels below minL are outside the window and have no bitset.  A
// grid-stride loop: each warp adds its count once at the end (one atomic per
// warp of a one-pass grid on the same counter serialised in L2).
__global__ void mark_deletions(const uint2* dels, uint64_t n, int L, int minL,
		uint32_t* const* del_words, unsigned long long* count) {
	unsigned long long c = 0;
	for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
			i += (uint64_t)gridDim.x * blockDim.x) {
		const uint2 d = dels[i];
		const uint32_t lv = d.y >> LG_BITS_LEVEL;
		const uint32_t ml = d.y & ((1u << LG_BITS_LEVEL) - 1u);
		if ((int)lv <= L && (int)lv >= minL && (int)ml <= L) {
			atomicOr(del_words[lv] + (d.x >> 5), 1u << (d.x & 31));
			c++;
		}
	}
#pragma unroll
	for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
	if ((threadIdx.x & 31u) == 0 && c) atomicAdd(count, c);
}

// lb[r] = first vertex e with pos[e] >= r * kBlockSlots (pos has V + 1
// entries), for r = 0..nb: the entry bounds of every PageRank block.
__global__ void block_lower_bounds(const uint32_t* pos, uint64_t V, uint64_t nb,
		uint32_t* lb) {
	const uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (r > nb) return;
	const uint64_t x = r * kBlockSlots;
	uint64_t lo = 0, hi = V;                     // answer in [lo, hi]
	while (lo < hi) {
		const uint64_t mid = (lo + hi) >> 1;
		if (pos[mid] < x) lo = mid + 1; else hi = mid;
	}
	lb[r] = (uint32_t)lo;
}

__global__ void sum_u32(const uint32_t* x, uint64_t n, unsigned long long* out) {
	unsigned long long s = 0;
	for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
			i += (uint64_t)gridDim.x * blockDim.x)
		s += x[i];
	for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
	if ((threadIdx.x & 31) == 0) atomicAdd(out, s);
}

static lg_status open_dir(lg_snapshot* sn, DevCsr& csr, SnapDir& d) {
	lg_store* s = sn->store;
	const int L = sn->level;
	SnapDir*& spare = s->snap_spare[&csr == &s->out ? 0 : 1];
	if (spare) d.swap_buffers(*spare);       // a closed snapshot's device buffers
	const int minL = sn->min_level;
	const uint64_t V = csr.levels[L]->max_nodes;
	cudaStream_t st = s->stream;
	VtTab tab;
	std::memset(&tab, 0, sizeof(tab));
	for (int l = minL; l <= L; l++) {
		tab.vt[l] = csr.levels[l]->vt.as<lg_vt_entry>();
		tab.max_nodes[l] = csr.levels[l]->max_nodes;
	}
	DevBuf& cnt = d.tmp_cnt;
	DevBuf& slots = d.tmp_slots;
	DevBuf& scan_tmp = d.tmp_scan;
	LG_TRY(cnt.reserve(V * sizeof(uint32_t)));
	LG_TRY(slots.reserve(V * sizeof(uint32_t)));
	LG_TRY(d.deg.reserve(V * sizeof(uint32_t)));
	LG_TRY(d.frag_off.reserve((V + 1) * sizeof(uint32_t)));
	const unsigned B = 256;
	walk_fragments<false><<<grid_for(V, B), B, 0, st>>>(tab, L, minL, V,
			cnt.as<uint32_t>(), d.deg.as<uint32_t>(), slots.as<uint32_t>(),
			nullptr, nullptr);
	LG_CUDA(cudaGetLastError(), "walk_fragments");
	s->launches += 5;   // two walks and the three scan kernels
	uint64_t F = 0;
	LG_TRY(exclusive_scan_u32(cnt.as<uint32_t>(), d.frag_off.as<uint32_t>(), V,
			scan_tmp, st, &F));
	d.n_frags = F;
	LG_TRY(d.frags.reserve(std::max<uint64_t>(F, 1) * sizeof(uint2)));
	walk_fragments<true><<<grid_for(V, B), B, 0, st>>>(tab, L, minL, V, nullptr,
			nullptr, nullptr, d.frag_off.as<uint32_t>(), d.frags.as<uint2>());
	LG_CUDA(cudaGetLastError(), "walk_fragments fill");

	// deletion bitsets of levels minL..L
	std::vector<uint64_t> word_off(L + 2, 0);
	for (int l = 0; l <= L; l++)
		word_off[l + 1] = word_off[l]
			+ (l < minL ? 0 : (csr.levels[l]->n_slots + 31) / 32 + 1);
	LG_TRY(d.delbits.reserve(word_off[L + 1] * sizeof(uint32_t)));
	LG_CUDA(cudaMemsetAsync(d.delbits.p, 0, word_off[L + 1] * sizeof(uint32_t), st),
			"clear deletion bits");
	LevelTab lt;
	std::memset(&lt, 0, sizeof(lt));
	for (int l = minL; l <= L; l++) {
		lt.ids[l] = csr.levels[l]->ids.as<uint32_t>();
		lt.del[l] = d.delbits.as<uint32_t>() + word_off[l];
		lt.w[l] = csr.levels[l]->w.p ? csr.levels[l]->w.as<uint32_t>() : nullptr;
	}
	LG_TRY(d.lt.reserve(sizeof(LevelTab)));
	LG_CUDA(cudaMemcpyAsync(d.lt.p, &lt, sizeof(lt), cudaMemcpyHostToDevice, st),
			"level table");
	DevBuf& counters = d.tmp_sum;     // [0] live degree sum, [1] deletions visible at L
	LG_TRY(counters.reserve(2 * sizeof(unsigned long long)));
	LG_CUDA(cudaMemsetAsync(counters.p, 0, 2 * sizeof(unsigned long long), st), "memset");
	if (csr.n_dels_dev > 0) {
		DevBuf& words = d.tmp_words;
		LG_TRY(words.reserve(sizeof(uint32_t*) * LG_MAX_LEVELS));
		LG_CUDA(cudaMemcpyAsync(words.p, lt.del, sizeof(lt.del),
				cudaMemcpyHostToDevice, st), "deletion table");
		int sms = 148;
		cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->device);
		const unsigned mark_blocks = std::min<unsigned>(grid_for(csr.n_dels_dev, B),
				(unsigned)sms * 8u);
		mark_deletions<<<mark_blocks, B, 0, st>>>(
				csr.dels.as<uint2>(), csr.n_dels_dev, L, minL,
				(uint32_t* const*)words.p, counters.as<unsigned long long>() + 1);
		LG_CUDA(cudaGetLastError(), "mark_deletions");
		s->launches++;
	}
	if (minL > 0) {
		// the vertex table's degree counts edges of every level: in a window
		// the degree is the number of live slots the chain covers
		SnapCsr g;
		g.frag_off = d.frag_off.as<uint32_t>();
		g.frags = d.frags.as<uint2>();
		g.lt = d.lt.as<LevelTab>();
		g.deg = d.deg.as<uint32_t>();
		g.V = V;
		live_counts<<<grid_for(V, B), B, 0, st>>>(g, d.deg.as<uint32_t>());
		LG_CUDA(cudaGetLastError(), "window degrees");
		s->launches++;
	}

	// per-vertex slot prefix (the virtual slot space the balanced kernels cut
	// into ranges) and the live edge count
	uint64_t total_slots = 0;
	LG_TRY(d.slot_off.reserve((V + 1) * sizeof(uint32_t)));
	LG_TRY(exclusive_scan_u32(slots.as<uint32_t>(), d.slot_off.as<uint32_t>(), V,
			scan_tmp, st, &total_slots));
	{
		const uint64_t nb = std::max<uint64_t>(1, (total_slots + kBlockSlots - 1) / kBlockSlots);
		LG_TRY(d.range_lb.reserve((nb + 1) * sizeof(uint32_t)));
		block_lower_bounds<<<grid_for(nb + 1, B), B, 0, st>>>(d.slot_off.as<uint32_t>(), V,
				nb, d.range_lb.as<uint32_t>());
		LG_CUDA(cudaGetLastError(), "block_lower_bounds");
		s->launches++;
	}
	sum_u32<<<592, B, 0, st>>>(d.deg.as<uint32_t>(), V, counters.as<unsigned long long>());
	LG_CUDA(cudaGetLastError(), "degree sum");
	s->launches += 4;
	unsigned long long sums[2] = {0, 0};
	LG_CUDA(cudaMemcpyAsync(sums, counters.p, sizeof(sums), cudaMemcpyDeviceToHost, st), "d2h");
	LG_CUDA(cudaStreamSynchronize(st), "snapshot sizes");
	d.n_edges = sums[0];
	d.n_frag_slots = total_slots;
	d.n_slots = 0;
	for (int l = minL; l <= L; l++) d.n_slots += csr.levels[l]->n_slots;
	d.n_dels = sums[1];
	d.present = true;
	return LG_OK;
}

// ---------------------------------------------------------------------------
// Adjacency materialisation (iteration order)
// ---------------------------------------------------------------------------

__global__ void live_counts(SnapCsr g, uint32_t* out) {
	uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (v >= g.V) return;
	uint32_t f0 = g.frag_off[v], f1 = g.frag_off[v + 1], c = 0;
	for (uint32_t f = f0; f < f1; f++) {
		uint2 fr = g.frags[f];
		uint32_t lv = frag_level(fr);
		for (uint32_t k = 0; k < frag_len(fr); k++)
			c += !slot_deleted(g.lt, lv, fr.x + k);
	}
	out[v] = c;
}

__global__ void write_adjacency(SnapCsr g, const uint32_t* off32,
		const unsigned long long* off64, uint32_t* nbr, long long* eid) {
	uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (v >= g.V) return;
	uint64_t o = off64 ? off64[v] : off32[v];
	uint32_t f0 = g.frag_off[v], f1 = g.frag_off[v + 1];
	for (uint32_t f = f0; f < f1; f++) {
		uint2 fr = g.frags[f];
		uint32_t lv = frag_level(fr);
		for (uint32_t k = 0; k < frag_len(fr); k++) {
			uint32_t ix = fr.x + k;
			if (slot_deleted(g.lt, lv, ix)) continue;
			nbr[o] = g.lt->ids[lv][ix];
			if (eid) eid[o] = (long long)LG_EDGE_CREATE(lv, ix);
			o++;
		}
	}
}

__global__ void widen_offsets(const uint32_t* cnt, uint64_t n,
		unsigned long long* out) {
	// single-CTA exclusive scan into 64-bit offsets
	unsigned long long carry = 0;
	for (uint64_t b = 0; b < n; b += blockDim.x) {
		uint64_t i = b + threadIdx.x;
		uint64_t x = i < n ? cnt[i] : 0, tot;
		uint64_t ex = block_excl_scan(x, &tot);
		if (i < n) out[i] = carry + ex;
		carry += tot;
	}
	if (threadIdx.x == 0) out[n] = carry;
}

} // namespace lg

using namespace lg;

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------

extern "C" {

size_t lg_last_error(char* buf, size_t len) {
	size_t n = strlen(t_err);
	if (buf && len) {
		size_t c = std::min(n, len - 1);
		std::memcpy(buf, t_err, c);
		buf[c] = 0;
	}
	return n;
}

const char* lg_status_string(lg_status st) {
	switch (st) {
	case LG_OK: return "ok";
	case LG_EINVAL: return "invalid argument";
	case LG_ENOMEM: return "out of memory";
	case LG_ECUDA: return "CUDA error";
	case LG_ETIMEOUT: return "timeout";
	case LG_ESTATE: return "invalid state";
	case LG_ENOTSUP: return "not supported";
	default: return "unknown status";
	}
}

const char* lg_version(void) { return "0.1.0"; }

lg_status lg_store_create(lg_store** out, const lg_store_opts* opts) {
	clear_error();
	if (!out) return set_error(LG_EINVAL, "null output pointer");
	*out = nullptr;
	int dev = opts ? opts->device : 0;
	int n = 0;
	cudaError_t e = cudaGetDeviceCount(&n);
	if (e != cudaSuccess || n == 0) {
		(void)cudaGetLastError();
		return set_error(LG_ECUDA, "no CUDA device available: %s",
				e == cudaSuccess ? "device count is 0" : cudaGetErrorString(e));
	}
	if (dev < 0 || dev >= n) return set_error(LG_EINVAL, "bad device ordinal %d", dev);
	LG_CUDA(cudaSetDevice(dev), "cudaSetDevice");
	lg_store* s = new (std::nothrow) lg_store();
	if (!s) return set_error(LG_ENOMEM, "host allocation");
	s->device = dev;
	s->reverse = opts ? opts->reverse_edges != 0 : true;
	if (opts && opts->stream) {
		s->stream = (cudaStream_t)opts->stream;
	} else {
		e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
		if (e != cudaSuccess) { delete s; return cuda_status(e, "stream"); }
		s->own_stream = true;
	}
	*out = s;
	return LG_OK;
}

lg_status lg_store_destroy(lg_store* s) {
	clear_error();
	if (!s) return LG_OK;
	if (s->open_snapshots > 0)
		return set_error(LG_ESTATE, "close all snapshots before destroying the store");
	cudaSetDevice(s->device);
	cudaStreamSynchronize(s->stream);
	if (s->copy_stream) {
		cudaStreamSynchronize(s->copy_stream);
		cudaStreamDestroy(s->copy_stream);
	}
	for (int i = 0; i < 2; i++) {
		if (s->staged[i]) cudaEventDestroy(s->staged[i]);
		if (s->stage_ready[i]) cudaEventDestroy(s->stage_ready[i]);
		if (s->stage_done[i]) cudaEventDestroy(s->stage_done[i]);
	}
	if (s->pinned) cudaFreeHost(s->pinned);
	if (s->host_words) cudaFreeHost(s->host_words);
	delete s->flat_scratch;
	for (int d = 0; d < 2; d++) {
		delete s->flat_spare[d];
		delete s->snap_spare[d];
		delete s->level_spare[d];
	}
	if (s->own_stream) cudaStreamDestroy(s->stream);
	delete s;
	return LG_OK;
}

lg_status lg_store_ingest_level(lg_store* s, const lg_level_desc* d) {
	clear_error();
	if (!s || !d) return set_error(LG_EINVAL, "null argument");
	LG_CUDA(cudaSetDevice(s->device), "cudaSetDevice");
	int l = (int)s->out.levels.size();
	if (l >= LG_MAX_LEVELS) return set_error(LG_ENOTSUP, "more than %d levels", LG_MAX_LEVELS);
	bool has_in = d->in.vt || d->in.vt_pages;
	if (s->reverse && !has_in)
		return set_error(LG_EINVAL, "store keeps reverse edges but the level has no in-CSR");
	if (s->reverse && d->in.max_nodes != d->out.max_nodes)
		return set_error(LG_EINVAL, "out and in CSR disagree on max_nodes");
	if (l > 0 && d->out.max_nodes < s->out.levels[l - 1]->max_nodes)
		return set_error(LG_EINVAL, "max_nodes cannot shrink");
	try {
		LG_TRY(ingest_csr(s, s->out, l, d->out, d->out_deletions,
				d->n_out_deletions, "out"));
		if (s->reverse) {
			lg_status st = ingest_csr(s, s->in, l, d->in, d->in_deletions,
					d->n_in_deletions, "in");
			if (st) {   // keep both directions at the same number of levels
				cudaStreamSynchronize(s->stream);
				delete s->out.levels.back();
				s->out.levels.pop_back();
				return st;
			}
		}
	} catch (const std::bad_alloc&) {
		return set_error(LG_ENOMEM, "host allocation during ingest");
	}
	LG_CUDA(cudaStreamSynchronize(s->stream), "ingest");
	return LG_OK;
}

int lg_store_num_levels(const lg_store* s) {
	return s ? (int)s->out.levels.size() : 0;
}

lg_status lg_store_max_nodes(const lg_store* s, int level, uint64_t* mn) {
	clear_error();
	if (!s || !mn) return set_error(LG_EINVAL, "null argument");
	if (level < 0) level = (int)s->out.levels.size() - 1;
	if (level < 0 || level >= (int)s->out.levels.size())
		return set_error(LG_EINVAL, "no such level");
	*mn = s->out.levels[level]->max_nodes;
	return LG_OK;
}

lg_status lg_store_sync(lg_store* s) {
	clear_error();
	if (!s) return set_error(LG_EINVAL, "null store");
	if (s->copy_stream) {
		// the store's stream waits for the result copies, so that work
		// queued on it after this call (an event, say) comes after them too
		for (int i = 0; i < 2; i++)
			LG_CUDA(cudaStreamWaitEvent(s->stream, s->stage_done[i], 0), "join copies");
		LG_CUDA(cudaStreamSynchronize(s->copy_stream), "sync copies");
	}
	LG_CUDA(cudaStreamSynchronize(s->stream), "sync");
	return LG_OK;
}

lg_status lg_store_set_output_mode(lg_store* s, int mode) {
	clear_error();
	if (!s) return set_error(LG_EINVAL, "null store");
	if (mode != LG_OUTPUT_SYNC && mode != LG_OUTPUT_ASYNC)
		return set_error(LG_EINVAL, "unknown output mode %d", mode);
	if (mode == LG_OUTPUT_SYNC && s->copy_stream)
		LG_CUDA(cudaStreamSynchronize(s->copy_stream), "sync copies");
	s->output_mode = mode;
	return LG_OK;
}

void* lg_store_stream(const lg_store* s) { return s ? (void*)s->stream : nullptr; }

uint64_t lg_store_device_bytes(const lg_store* s) {
	if (!s) return 0;
	uint64_t b = 0;
	for (const DevCsr* c : {&s->out, &s->in}) {
		for (const DevLevel* l : c->levels) b += l->vt.bytes + l->ids.bytes + l->w.bytes;
		b += c->dels.bytes;
	}
	for (const DevBuf& x : s->scratch) b += x.bytes;
	return b;
}

uint64_t lg_store_launch_count(const lg_store* s) { return s ? s->launches : 0; }

lg_status lg_store_transfer_bytes(const lg_store* s, uint64_t* h2d, uint64_t* d2h) {
	clear_error();
	if (!s) return set_error(LG_EINVAL, "null store");
	if (h2d) *h2d = s->h2d_bytes;
	if (d2h) *d2h = s->d2h_bytes;
	return LG_OK;
}

lg_status lg_store_drop_level(lg_store* s) {
	clear_error();
	if (!s) return set_error(LG_EINVAL, "null store");
	if (s->out.levels.empty()) return set_error(LG_ESTATE, "the store holds no level");
	if (s->open_snapshots > 0)
		return set_error(LG_ESTATE, "close all snapshots before dropping a level");
	if ((int)s->out.levels.size() - 1 <= s->min_level && s->min_level > 0)
		return set_error(LG_ESTATE, "the newest level is the only one not aged out");
	LG_CUDA(cudaSetDevice(s->device), "cudaSetDevice");
	LG_CUDA(cudaStreamSynchronize(s->stream), "drop level");
	for (int dir = 0; dir < 2; dir++) {
		DevCsr* c = dir == 0 ? &s->out : &s->in;
		if (c->levels.empty()) continue;
		delete s->level_spare[dir];               // keep the newest dropped level's buffers
		s->level_spare[dir] = c->levels.back();
		c->levels.pop_back();
		// the list keeps the marks of the levels below
		c->n_dels_dev = c->dels_mark.back();
		c->dels_mark.pop_back();
	}
	return LG_OK;
}

lg_status lg_snapshot_get_stats(const lg_snapshot* sn, int dir, lg_snapshot_stats* st) {
	clear_error();
	if (!sn || !st) return set_error(LG_EINVAL, "null argument");
	if (dir != 0 && dir != 1) return set_error(LG_EINVAL, "dir must be 0 or 1");
	const SnapDir& d = dir == 0 ? sn->out : sn->in;
	if (!d.present) return set_error(LG_ESTATE, "the store has no in-CSR");
	st->max_nodes = sn->V;
	st->live_edges = d.n_edges;
	st->slots = d.n_slots;
	st->fragment_slots = d.n_frag_slots;
	st->fragments = d.n_frags;
	st->ranges = (d.n_frag_slots + kBlockSlots - 1) / kBlockSlots;
	st->deletions = d.n_dels;
	return LG_OK;
}

lg_status lg_snapshot_open_window(lg_store* s, int level, int min_level,
		lg_snapshot** out) {
	clear_error();
	if (!s || !out) return set_error(LG_EINVAL, "null argument");
	*out = nullptr;
	int n = (int)s->out.levels.size();
	if (level < 0) level = n - 1;
	if (level < 0 || level >= n) return set_error(LG_EINVAL, "no such level %d", level);
	if (min_level < s->min_level || min_level > level)
		return set_error(LG_EINVAL, "min_level %d outside [%d, %d] (levels below %d are "
				"aged out)", min_level, s->min_level, level, s->min_level);
	LG_CUDA(cudaSetDevice(s->device), "cudaSetDevice");
	lg_snapshot* sn = new (std::nothrow) lg_snapshot();
	if (!sn) return set_error(LG_ENOMEM, "host allocation");
	sn->store = s;
	sn->level = level;
	sn->min_level = min_level;
	sn->V = s->out.levels[level]->max_nodes;
	lg_status st = open_dir(sn, s->out, sn->out);
	if (!st && s->reverse) st = open_dir(sn, s->in, sn->in);
	if (st) { cudaStreamSynchronize(s->stream); delete sn; return st; }
	s->open_snapshots++;
	*out = sn;
	return LG_OK;
}

lg_status lg_snapshot_open(lg_store* s, int level, lg_snapshot** out) {
	if (!s) { clear_error(); return set_error(LG_EINVAL, "null argument"); }
	int lv = level < 0 ? (int)s->out.levels.size() - 1 : level;
	if (lv >= 0 && lv < s->min_level) {
		clear_error();
		return set_error(LG_EINVAL, "level %d is aged out (min level %d)", lv, s->min_level);
	}
	return lg_snapshot_open_window(s, level, s->min_level, out);
}

lg_status lg_snapshot_min_level(const lg_snapshot* sn, int* min_level) {
	if (!sn || !min_level) return set_error(LG_EINVAL, "null argument");
	*min_level = sn->min_level;
	return LG_OK;
}

lg_status lg_store_set_min_level(lg_store* s, int m) {
	clear_error();
	if (!s) return set_error(LG_EINVAL, "null store");
	const int n = (int)s->out.levels.size();
	if (m < s->min_level) return set_error(LG_EINVAL, "the min level cannot decrease");
	if (m > n - 1) return set_error(LG_EINVAL, "min level %d would age out every level", m);
	if (s->open_snapshots > 0)
		return set_error(LG_ESTATE, "close all snapshots before aging levels out");
	LG_CUDA(cudaSetDevice(s->device), "cudaSetDevice");
	LG_CUDA(cudaStreamSynchronize(s->stream), "set min level");
	for (int l = s->min_level; l < m; l++) {
		for (DevCsr* c : {&s->out, &s->in}) {
			if (l >= (int)c->levels.size()) continue;
			DevLevel* d = c->levels[l];
			d->vt.release();       // sizes (max_nodes, n_slots) stay for validation
			d->ids.release();
			d->w.release();
		}
	}
	s->min_level = m;
	return LG_OK;
}

int lg_store_min_level(const lg_store* s) { return s ? s->min_level : 0; }

lg_status lg_snapshot_close(lg_snapshot* sn) {
	clear_error();
	if (!sn) return LG_OK;
	cudaSetDevice(sn->store->device);
	cudaStreamSynchronize(sn->store->stream);
	sn->store->open_snapshots--;
	if (sn->adj_maps) lg_free_adjoint_maps(sn->adj_maps);
	if (sn->sssp_split) lg_free_sssp_split(sn->sssp_split);
	for (int d = 0; d < 2; d++) lg_flat_release(sn->store, sn->flat[d]);
	// keep this snapshot's device buffers for the next open
	lg_store* s = sn->store;
	for (int d = 0; d < 2; d++) {
		SnapDir& sd = d == 0 ? sn->out : sn->in;
		if (!sd.present) continue;
		if (!s->snap_spare[d]) s->snap_spare[d] = new (std::nothrow) SnapDir();
		if (s->snap_spare[d]) s->snap_spare[d]->swap_buffers(sd);
	}
	delete sn;
	return LG_OK;
}

lg_status lg_snapshot_level(const lg_snapshot* sn, int* level) {
	if (!sn || !level) return set_error(LG_EINVAL, "null argument");
	*level = sn->level;
	return LG_OK;
}

lg_status lg_snapshot_max_nodes(const lg_snapshot* sn, uint64_t* mn) {
	if (!sn || !mn) return set_error(LG_EINVAL, "null argument");
	*mn = sn->V;
	return LG_OK;
}

lg_status lg_snapshot_num_edges(const lg_snapshot* sn, uint64_t* ne) {
	if (!sn || !ne) return set_error(LG_EINVAL, "null argument");
	*ne = sn->out.n_edges;
	return LG_OK;
}

static lg_status degrees(lg_snapshot* sn, int dir, uint32_t* out) {
	clear_error();
	if (!sn || !out) return set_error(LG_EINVAL, "null argument");
	const SnapDir& d = dir == 0 ? sn->out : sn->in;
	if (!d.present) return set_error(LG_ESTATE, "the store has no in-CSR");
	lg_store* s = sn->store;
	LG_CUDA(cudaSetDevice(s->device), "cudaSetDevice");
	LG_TRY(copy_out(s, out, d.deg.p, sn->V * sizeof(uint32_t)));
	LG_CUDA(cudaStreamSynchronize(s->stream), "degrees");
	return LG_OK;
}

lg_status lg_out_degrees(lg_snapshot* sn, uint32_t* out) { return degrees(sn, 0, out); }
lg_status lg_in_degrees(lg_snapshot* sn, uint32_t* out) { return degrees(sn, 1, out); }

lg_status lg_snapshot_adjacency(lg_snapshot* sn, int dir, uint64_t* offsets,
		uint32_t* neighbors, int64_t* edge_ids) {
	clear_error();
	if (!sn || !offsets) return set_error(LG_EINVAL, "null argument");
	if (dir != 0 && dir != 1) return set_error(LG_EINVAL, "dir must be 0 or 1");
	const SnapDir& d = dir == 0 ? sn->out : sn->in;
	if (!d.present) return set_error(LG_ESTATE, "the store has no in-CSR");
	lg_store* s = sn->store;
	LG_CUDA(cudaSetDevice(s->device), "cudaSetDevice");
	cudaStream_t st = s->stream;
	SnapCsr g = sn->view(dir);
	const uint64_t V = sn->V;
	DevBuf cnt, off, nb, ei;
	LG_TRY(cnt.reserve(V * 4));
	LG_TRY(off.reserve((V + 1) * 8));
	live_counts<<<grid_for(V, 256), 256, 0, st>>>(g, cnt.as<uint32_t>());
	widen_offsets<<<1, 1024, 0, st>>>(cnt.as<uint32_t>(), V,
			off.as<unsigned long long>());
	LG_CUDA(cudaGetLastError(), "adjacency offsets");
	s->launches += 3;
	uint64_t E = 0;
	LG_CUDA(cudaMemcpyAsync(&E, off.as<unsigned long long>() + V, 8,
			cudaMemcpyDeviceToHost, st), "d2h");
	LG_CUDA(cudaStreamSynchronize(st), "adjacency");
	LG_TRY(nb.reserve(std::max<uint64_t>(E, 1) * 4));
	if (edge_ids) LG_TRY(ei.reserve(std::max<uint64_t>(E, 1) * 8));
	write_adjacency<<<grid_for(V, 256), 256, 0, st>>>(g, nullptr,
			off.as<unsigned long long>(), nb.as<uint32_t>(),
			edge_ids ? ei.as<long long>() : nullptr);
	LG_CUDA(cudaGetLastError(), "write_adjacency");
	LG_TRY(copy_out(s, offsets, off.p, (V + 1) * 8));
	if (neighbors) LG_TRY(copy_out(s, neighbors, nb.p, E * 4));
	if (edge_ids) LG_TRY(copy_out(s, edge_ids, ei.p, E * 8));
	LG_CUDA(cudaStreamSynchronize(st), "adjacency");
	return LG_OK;
}

} // extern "C"
