// lg_device.cuh - device mirror of a LLAMA level stack and the warp-level
// traversal primitive every analytics kernel is built on.
//
// Layout in HBM (one per CSR direction):
//   level l:  vt[l]      (max_nodes_l + 1) x 16 B vertex-table elements, the
//                        flattened copy-on-write table of that level
//             ids[l]     n_slots_l x u32 neighbour ids; slots that are not
//                        part of a fragment (continuation records, unused
//                        continuation space) hold 0xffffffff and are never read
//             w[l]       optional n_slots_l x u32 edge property
//   deletions            every slot whose max_visible_level was lowered, as
//                        (index, level << 26 | max_visible_level)
// A snapshot L adds, per direction:
//   frag_off   (V + 1) x u32   prefix of per-vertex fragment counts
//   frags      F x uint2       {slot index, len << 6 | level}: the vertex's
//                              continuation chain resolved newest-first
//   del[l]     bitset over level l's slots, bit = max_visible_level <= L
//   deg        V x u32         live degree (the vertex-table degree field)
//   slot_off   (V + 1) x u32   prefix of per-vertex fragment lengths: the
//                              virtual slot space balanced kernels cut up
#ifndef LG_DEVICE_CUH_
#define LG_DEVICE_CUH_

#include <cuda_runtime.h>
#include <stdint.h>

#include <utility>
#include <vector>

#include "lg_internal.h"

namespace lg {

constexpr uint32_t kNoId = 0xffffffffu;
constexpr int kLevelBits = 6;                 // level field of a fragment
constexpr uint32_t kLevelMask = (1u << kLevelBits) - 1u;

// Per-snapshot, per-direction table of level base pointers.
struct LevelTab {
	const uint32_t* ids[LG_MAX_LEVELS];
	const uint32_t* del[LG_MAX_LEVELS];
	const uint32_t* w[LG_MAX_LEVELS];
};

// What a kernel needs to walk one direction of a snapshot.
struct SnapCsr {
	const uint32_t* frag_off;   // V + 1
	const uint2* frags;         // F
	const LevelTab* lt;         // device copy
	const uint32_t* deg;        // V
	uint64_t V;
};

__device__ __forceinline__ uint32_t frag_len(uint2 f) { return f.y >> kLevelBits; }
__device__ __forceinline__ uint32_t frag_level(uint2 f) { return f.y & kLevelMask; }

__device__ __forceinline__ bool slot_deleted(const LevelTab* lt, uint32_t lv,
		uint32_t idx) {
	const uint32_t* d = lt->del[lv];
	return (__ldg(d + (idx >> 5)) >> (idx & 31)) & 1u;
}

// Slots (live or deleted) of vertex v's fragments in this snapshot.
__device__ __forceinline__ uint32_t vertex_slots(const SnapCsr& g, uint32_t v,
		uint32_t* f0out) {
	uint32_t f0 = __ldg(g.frag_off + v), f1 = __ldg(g.frag_off + v + 1);
	uint32_t c = 0;
	for (uint32_t f = f0; f < f1; f++) c += frag_len(g.frags[f]);
	*f0out = f0;
	return c;
}

// Warp-cooperative expansion.  Every lane brings one vertex (`cnt` slots
// starting at fragment `f0`, cnt = 0 for none); the warp walks the union of
// those slots 32 at a time, lane k taking the k-th slot of the chunk, so the
// neighbour-id loads of a chunk are contiguous within each fragment.  For
// every chunk `body(active, owner_lane, nbr, level, index)` runs on all 32
// lanes (active = the lane holds a live slot), so the body may use warp
// collectives.  Owners are non-decreasing across the lanes of a chunk.
template <class Body>
__device__ __forceinline__ void warp_expand(const SnapCsr& g, uint32_t cnt,
		uint32_t f0, Body&& body) {
	const uint32_t lane = threadIdx.x & 31u;
	uint32_t incl = cnt;
#pragma unroll
	for (int o = 1; o < 32; o <<= 1) {
		uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
		if (lane >= (uint32_t)o) incl += t;
	}
	const uint32_t excl = incl - cnt;
	const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
	for (uint32_t base = 0; base < total; base += 32) {
		const uint32_t k = base + lane;
		// owner = last lane whose range starts at or before k
		uint32_t o = 0;
#pragma unroll
		for (uint32_t step = 16; step > 0; step >>= 1) {
			uint32_t cand = o + step;
			uint32_t e = __shfl_sync(0xffffffffu, excl, cand & 31u);
			if (cand < 32 && e <= k) o = cand;
		}
		const uint32_t oexcl = __shfl_sync(0xffffffffu, excl, o);
		uint32_t f = __shfl_sync(0xffffffffu, f0, o);
		bool act = k < total;
		uint32_t nbr = kNoId, lv = 0, idx = 0;
		if (act) {
			uint32_t r = k - oexcl;
			uint2 fr = g.frags[f];
			while (r >= frag_len(fr)) { r -= frag_len(fr); fr = g.frags[++f]; }
			lv = frag_level(fr);
			idx = fr.x + r;
			act = !slot_deleted(g.lt, lv, idx);
			if (act) nbr = __ldg(g.lt->ids[lv] + idx);
		}
		body(act, o, nbr, lv, idx);
	}
}

// Warp inclusive segmented sum of `v` over lanes with equal `key` (keys are
// non-decreasing); returns the sum at each lane and sets *tail for the last
// lane of every segment.
__device__ __forceinline__ double warp_segsum(double v, uint32_t key, bool* tail) {
	const uint32_t lane = threadIdx.x & 31u;
#pragma unroll
	for (int o = 1; o < 32; o <<= 1) {
		double t = __shfl_up_sync(0xffffffffu, v, o);
		uint32_t k = __shfl_up_sync(0xffffffffu, key, o);
		if (lane >= (uint32_t)o && k == key) v += t;
	}
	uint32_t nk = __shfl_down_sync(0xffffffffu, key, 1);
	*tail = (lane == 31u) || (nk != key);
	return v;
}

// ---------------------------------------------------------------------------
// Host-side objects
// ---------------------------------------------------------------------------

// Device allocation owned by a host object.
struct DevBuf {
	void* p = nullptr;
	size_t bytes = 0;
	DevBuf() = default;
	DevBuf(const DevBuf&) = delete;
	DevBuf& operator=(const DevBuf&) = delete;
	~DevBuf() { release(); }
	void release() { if (p) cudaFree(p); p = nullptr; bytes = 0; }
	// (Re)allocate to at least n bytes; contents are not preserved.
	lg_status reserve(size_t n);
	template <class T> T* as() const { return static_cast<T*>(p); }
	void swap(DevBuf& o) { std::swap(p, o.p); std::swap(bytes, o.bytes); }
};

struct DevLevel {
	uint64_t max_nodes = 0;
	uint64_t n_slots = 0;
	uint64_t n_fragment_slots = 0;   // slots that belong to this level's fragments
	DevBuf vt;        // lg_vt_entry[max_nodes + 1]
	DevBuf ids;       // u32[n_slots]
	DevBuf w;         // u32[n_slots] or empty
};

struct DevCsr {
	std::vector<DevLevel*> levels;
	// deletion marks (index, level << 26 | max_visible_level) of all levels,
	// in level order, on the device only
	DevBuf dels;
	uint64_t n_dels_dev = 0;        // marks in dels
	std::vector<size_t> dels_mark;  // n_dels_dev before each level's marks
	~DevCsr() { for (DevLevel* l : levels) delete l; }
};

// Slots per PageRank block; range_lb below is computed for this size.
constexpr uint32_t kBlockSlots = 1024;

struct SnapDir {
	DevBuf frag_off, frags, deg, delbits, lt, slot_off;
	DevBuf range_lb;               // lower_bound(slot_off, r * kBlockSlots), r = 0..nblocks
	DevBuf tmp_cnt, tmp_slots, tmp_scan, tmp_words, tmp_sum;   // open-time scratch
	uint64_t n_frags = 0;
	uint64_t n_edges = 0;          // live edges (sum of degrees)
	uint64_t n_slots = 0;          // slots of levels 0..L
	uint64_t n_frag_slots = 0;     // slots covered by fragments
	uint64_t n_dels = 0;           // deletion marks visible at L
	bool present = false;
	// exchange device buffers with o (a closed snapshot's, kept for reuse)
	void swap_buffers(SnapDir& o) {
		DevBuf* a[] = {&frag_off, &frags, &deg, &delbits, &lt, &slot_off, &range_lb,
			&tmp_cnt, &tmp_slots, &tmp_scan, &tmp_words, &tmp_sum};
		DevBuf* b[] = {&o.frag_off, &o.frags, &o.deg, &o.delbits, &o.lt, &o.slot_off,
			&o.range_lb, &o.tmp_cnt, &o.tmp_slots, &o.tmp_scan, &o.tmp_words, &o.tmp_sum};
		for (size_t i = 0; i < sizeof(a) / sizeof(a[0]); i++) a[i]->swap(*b[i]);
	}
	SnapCsr view() const {
		SnapCsr s;
		s.frag_off = frag_off.as<uint32_t>();
		s.frags = frags.as<uint2>();
		s.lt = lt.as<LevelTab>();
		s.deg = deg.as<uint32_t>();
		s.V = 0;
		return s;
	}
};

struct FlatCsr;   // lg_flat.cuh

} // namespace lg

struct lg_store {
	int device = 0;
	cudaStream_t stream = nullptr;
	bool own_stream = false;
	bool reverse = false;
	lg::DevCsr out, in;
	// pinned staging for host -> device copies (two halves, double-buffered)
	void* pinned = nullptr;
	size_t pinned_bytes = 0;
	// a few pinned words for per-step counters read back by the host loops
	unsigned long long* host_words = nullptr;
	cudaEvent_t staged[2] = {nullptr, nullptr};
	// scratch shared by the analytics calls of this store
	lg::DevBuf scratch[12];
	int open_snapshots = 0;
	uint64_t launches = 0;      // kernels launched by this store
	uint64_t h2d_bytes = 0;     // host -> device bytes copied by this store
	uint64_t d2h_bytes = 0;     // device -> host bytes copied by this store
	lg::FlatCsr* flat_scratch = nullptr;   // per-call flat in-CSR of PageRank
	lg::FlatCsr* flat_spare[2] = {nullptr, nullptr};   // unflattened, kept for reuse
	// device buffers of the last closed snapshot and the last dropped level,
	// per direction, reused by the next open / level (the stream was
	// synchronised when they were released)
	lg::SnapDir* snap_spare[2] = {nullptr, nullptr};
	lg::DevLevel* level_spare[2] = {nullptr, nullptr};
	lg::DevBuf build_tmp[12];   // lg_store_build_level temporaries
	int min_level = 0;          // levels below are aged out (lg_store_set_min_level)
	// LG_OUTPUT_ASYNC: results staged in out_stage[i] and copied to host on
	// copy_stream; stage_done[i] marks the end of slot i's last copy
	int output_mode = 0;
	cudaStream_t copy_stream = nullptr;
	lg::DevBuf out_stage[2];
	cudaEvent_t stage_ready[2] = {nullptr, nullptr};
	cudaEvent_t stage_done[2] = {nullptr, nullptr};
	int stage_next = 0;
};

// Edge-order maps of a snapshot used by the differentiable PageRank
// (lg_adjoint.cu); built on first use, freed with the snapshot.
struct lg_adjoint_maps;
void lg_free_adjoint_maps(lg_adjoint_maps* m);

// The snapshot's out-edges split by weight for delta-stepping (lg_sssp.cu);
// built on first use for a delta, freed with the snapshot.
struct lg_sssp_split;
void lg_free_sssp_split(lg_sssp_split* p);

struct lg_snapshot {
	lg_store* store = nullptr;
	lg_adjoint_maps* adj_maps = nullptr;
	lg_sssp_split* sssp_split = nullptr;
	lg::FlatCsr* flat[2] = {nullptr, nullptr};   // lg_snapshot_flatten, per direction
	int level = 0;
	int min_level = 0;          // oldest level the snapshot sees
	uint64_t V = 0;
	lg::SnapDir out, in;
	lg::SnapCsr view(int dir) const {
		lg::SnapCsr s = (dir == 0 ? out : in).view();
		s.V = V;
		return s;
	}
};

namespace lg {

// CUDA error -> lg_status with a message naming the failing step.
lg_status cuda_status(cudaError_t e, const char* what);
#define LG_CUDA(call, what) do { cudaError_t _e = (call); \
	if (_e != cudaSuccess) return ::lg::cuda_status(_e, what); } while (0)
#define LG_TRY(expr) do { lg_status _s = (expr); if (_s) return _s; } while (0)

// True if p is device (or managed) memory usable by the store's GPU.
bool is_device_pointer(const void* p);

// Exclusive scan of n u32 counts into out[0..n] (u32); returns false if the
// total does not fit 32 bits.  Runs on `stream`, uses `tmp` as scratch.
lg_status exclusive_scan_u32(const uint32_t* in, uint32_t* out, uint64_t n,
		DevBuf& tmp, cudaStream_t stream, uint64_t* total);

// Copy `bytes` of device data to a caller buffer (host or device) on the
// store's stream, counting host-bound bytes.
lg_status copy_out(lg_store* s, void* dst, const void* src, size_t bytes);

// The store's kHostWords pinned words (allocated on first use), for
// counters a host loop reads back every step.
constexpr int kHostWords = 16;
lg_status host_words(lg_store* s, unsigned long long** words);
// Waits for the store's stream and reads n <= 8 device words into out through
// pinned words 8..15 (words 0..7 stay with the caller).
lg_status read_words(lg_store* s, const unsigned long long* dev, int n, unsigned long long* out);

// A DevLevel for direction dir (0 out, 1 in) of a new level: the store's
// spare (buffers of the last dropped level) or a new one.  Null if the host
// allocation fails.
DevLevel* take_level(lg_store* s, int dir);

// Appends a level's n deletion marks (host or device memory, per kind) to
// csr's device list and records where the level's marks begin.
lg_status append_dels(lg_store* s, DevCsr& csr, const uint2* add, size_t n,
		cudaMemcpyKind kind);

inline unsigned grid_for(uint64_t n, unsigned block) {
	uint64_t g = (n + block - 1) / block;
	return (unsigned)(g > 0x7fffffffull ? 0x7fffffffull : (g == 0 ? 1 : g));
}

} // namespace lg

#endif // LG_DEVICE_CUH_
