// lg_sort.cu - device LSD radix sort of 64-bit keys (optional 32-bit
// payload) and de-duplication, used to flatten and orient snapshots.
//
// One pass per 8-bit digit that varies over the input (the varying bits are
// found first with an OR/AND reduction, so 48-bit keys cost 6 passes):
//   rs_hist     per-tile digit counts, stored digit-major
//   scan        exclusive scan of the counts -> scatter bases
//   rs_scatter  stable scatter: a tile is ranked in 16 rounds of 256 keys;
//               inside a round, __match_any_sync groups the lanes of a warp
//               that share a digit and the per-warp counts in shared memory
//               give the rank across warps, so equal digits keep input order.
#include "lg_device.cuh"
#include "lg_sort.cuh"

namespace lg {

constexpr int kRsThreads = 256;
constexpr int kRsItems = 16;
constexpr uint64_t kRsTile = (uint64_t)kRsThreads * kRsItems;
constexpr int kRsWarps = kRsThreads / 32;

__global__ void rs_bits(const unsigned long long* k, uint64_t n,
		unsigned long long* or_and) {
	unsigned long long o = 0, a = ~0ull;
	for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
			i += (uint64_t)gridDim.x * blockDim.x) {
		o |= k[i];
		a &= k[i];
	}
	for (int s = 16; s > 0; s >>= 1) {
		o |= __shfl_down_sync(0xffffffffu, o, s);
		a &= __shfl_down_sync(0xffffffffu, a, s);
	}
	if ((threadIdx.x & 31) == 0) { atomicOr(or_and, o); atomicAnd(or_and + 1, a); }
}

__global__ void __launch_bounds__(kRsThreads)
rs_hist(const unsigned long long* k, uint64_t n, int shift, uint32_t* counts,
		uint32_t tiles) {
	__shared__ uint32_t h[256];
	h[threadIdx.x] = 0;
	__syncthreads();
	const uint64_t base = (uint64_t)blockIdx.x * kRsTile;
	for (int r = 0; r < kRsItems; r++) {
		uint64_t i = base + (uint64_t)r * kRsThreads + threadIdx.x;
		if (i < n) atomicAdd(&h[(k[i] >> shift) & 0xff], 1u);
	}
	__syncthreads();
	counts[(uint64_t)threadIdx.x * tiles + blockIdx.x] = h[threadIdx.x];
}

__global__ void __launch_bounds__(kRsThreads)
rs_scatter(const unsigned long long* k, const uint32_t* pin, uint64_t n, int shift,
		const uint32_t* offsets, uint32_t tiles, unsigned long long* kout,
		uint32_t* pout) {
	__shared__ uint32_t base[256];
	__shared__ uint32_t run[256];
	__shared__ uint32_t wcnt[kRsWarps][256];
	const uint32_t lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
	base[threadIdx.x] = offsets[(uint64_t)threadIdx.x * tiles + blockIdx.x];
	run[threadIdx.x] = 0;
	for (int x = 0; x < kRsWarps; x++) wcnt[x][threadIdx.x] = 0;
	__syncthreads();
	const uint64_t tile0 = (uint64_t)blockIdx.x * kRsTile;
	for (int r = 0; r < kRsItems; r++) {
		const uint64_t i = tile0 + (uint64_t)r * kRsThreads + threadIdx.x;
		const bool valid = i < n;
		unsigned long long key = valid ? k[i] : 0;
		uint32_t pay = (valid && pin) ? pin[i] : 0;
		// invalid lanes take digit 256, which matches no real digit
		const uint32_t dig = valid ? (uint32_t)((key >> shift) & 0xff) : 256u;
		const unsigned peers = __match_any_sync(0xffffffffu, dig);
		const uint32_t wrank = __popc(peers & ((1u << lane) - 1u));
		if (valid && (32 - __clz(peers)) - 1 == (int)lane) wcnt[w][dig] = __popc(peers);
		__syncthreads();
		if (valid) {
			uint32_t before = run[dig];
			for (uint32_t x = 0; x < w; x++) before += wcnt[x][dig];
			const uint32_t pos = base[dig] + before + wrank;
			kout[pos] = key;
			if (pout) pout[pos] = pay;
		}
		__syncthreads();
		{
			uint32_t t = 0;
			for (int x = 0; x < kRsWarps; x++) { t += wcnt[x][threadIdx.x]; wcnt[x][threadIdx.x] = 0; }
			run[threadIdx.x] += t;
		}
		__syncthreads();
	}
}

__global__ void mark_first(const unsigned long long* k, uint64_t n, uint32_t* flag) {
	uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n) flag[i] = (i == 0 || k[i] != k[i - 1]) ? 1u : 0u;
}

__global__ void compact_first(const unsigned long long* k, uint64_t n,
		const uint32_t* flag, const uint32_t* pos, unsigned long long* out) {
	uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n && flag[i]) out[pos[i]] = k[i];
}

lg_status radix_sort_u64(lg_store* s, unsigned long long* keys, uint32_t* payload,
		uint64_t n, DevBuf& tmp_keys, DevBuf& tmp_pay, DevBuf& counts, DevBuf& scan_tmp,
		unsigned long long** sorted_keys, uint32_t** sorted_pay) {
	cudaStream_t st = s->stream;
	*sorted_keys = keys;
	if (sorted_pay) *sorted_pay = payload;
	if (n < 2) return LG_OK;
	if (n >= 0xffffffffull) return set_error(LG_ENOTSUP, "sort of more than 2^32-1 keys");
	const uint32_t tiles = (uint32_t)((n + kRsTile - 1) / kRsTile);
	LG_TRY(tmp_keys.reserve(n * 8));
	if (payload) LG_TRY(tmp_pay.reserve(n * 4));
	LG_TRY(counts.reserve(((uint64_t)256 * tiles + 1) * 8 + 16));
	uint32_t* cnt = counts.as<uint32_t>();
	uint32_t* off = cnt + (uint64_t)256 * tiles + 1;
	// which bits vary
	unsigned long long oa[2] = {0, ~0ull};
	unsigned long long* d_oa = (unsigned long long*)(counts.as<char>()
			+ ((uint64_t)256 * tiles + 1) * 8);
	LG_CUDA(cudaMemcpyAsync(d_oa, oa, 16, cudaMemcpyHostToDevice, st), "h2d");
	rs_bits<<<592, 256, 0, st>>>(keys, n, d_oa);
	LG_CUDA(cudaMemcpyAsync(oa, d_oa, 16, cudaMemcpyDeviceToHost, st), "d2h");
	LG_CUDA(cudaStreamSynchronize(st), "sort bits");
	s->launches++;
	const unsigned long long vary = oa[0] ^ oa[1];
	unsigned long long* src = keys;
	unsigned long long* dst = tmp_keys.as<unsigned long long>();
	uint32_t* psrc = payload;
	uint32_t* pdst = payload ? tmp_pay.as<uint32_t>() : nullptr;
	for (int shift = 0; shift < 64; shift += 8) {
		if (((vary >> shift) & 0xff) == 0) continue;
		rs_hist<<<tiles, kRsThreads, 0, st>>>(src, n, shift, cnt, tiles);
		LG_TRY(exclusive_scan_u32(cnt, off, (uint64_t)256 * tiles, scan_tmp, st, nullptr));
		rs_scatter<<<tiles, kRsThreads, 0, st>>>(src, psrc, n, shift, off, tiles, dst, pdst);
		LG_CUDA(cudaGetLastError(), "radix sort pass");
		s->launches += 5;
		std::swap(src, dst);
		std::swap(psrc, pdst);
	}
	*sorted_keys = src;
	if (sorted_pay) *sorted_pay = psrc;
	return LG_OK;
}

lg_status unique_u64(lg_store* s, const unsigned long long* keys, uint64_t n,
		unsigned long long* out, DevBuf& flags, DevBuf& scan_tmp, uint64_t* n_out) {
	cudaStream_t st = s->stream;
	if (n == 0) { *n_out = 0; return LG_OK; }
	LG_TRY(flags.reserve((2 * n + 1) * 4));
	uint32_t* fl = flags.as<uint32_t>();
	uint32_t* pos = fl + n;
	mark_first<<<grid_for(n, 256), 256, 0, st>>>(keys, n, fl);
	uint64_t total = 0;
	LG_TRY(exclusive_scan_u32(fl, pos, n, scan_tmp, st, &total));
	compact_first<<<grid_for(n, 256), 256, 0, st>>>(keys, n, fl, pos, out);
	LG_CUDA(cudaGetLastError(), "unique");
	s->launches += 5;
	*n_out = total;
	return LG_OK;
}

} // namespace lg
