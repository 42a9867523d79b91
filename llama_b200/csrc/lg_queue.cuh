// lg_queue.cuh - appends to a device list from many warps without
// serialising on its length counter: per-warp staging in shared memory
// (wq_add / wq_flush) and a CTA-wide append (block_push).
#ifndef LG_QUEUE_CUH_
#define LG_QUEUE_CUH_

#include <cuda_runtime.h>
#include <stdint.h>

namespace lg {

// Per-warp staging of queue appends in shared memory: items collect in a
// kPushBuf-entry buffer and go to the global queue kPushBuf at a time with
// one atomic, instead of one atomic on the same counter per 32 items (which
// serialises in L2 when most warps append).  n is warp-uniform.
constexpr uint32_t kPushBuf = 128;

__device__ __forceinline__ void wq_flush(uint32_t* sbuf, uint32_t& n, uint32_t* queue,
		unsigned long long* len) {
	if (n == 0) return;
	const uint32_t lane = threadIdx.x & 31u;
	__syncwarp();
	unsigned long long base = 0;
	if (lane == 0) base = atomicAdd(len, (unsigned long long)n);
	base = __shfl_sync(0xffffffffu, base, 0);
	for (uint32_t i = lane; i < n; i += 32u) queue[base + i] = sbuf[i];
	__syncwarp();
	n = 0;
}

__device__ __forceinline__ void wq_add(bool take, uint32_t item, uint32_t* sbuf, uint32_t& n,
		uint32_t* queue, unsigned long long* len) {
	const unsigned m = __ballot_sync(0xffffffffu, take);
	if (!m) return;
	if (n + (uint32_t)__popc(m) > kPushBuf) wq_flush(sbuf, n, queue, len);
	const uint32_t lane = threadIdx.x & 31u;
	if (take) sbuf[n + __popc(m & ((1u << lane) - 1u))] = item;
	n += __popc(m);
}

// CTA-wide append: every thread of the CTA (kThreads of them) calls it with
// its (take, item); the CTA's items go to list at slots taken from *len with
// one atomic, in thread order.
template <int kThreads>
__device__ __forceinline__ void block_push(bool take, uint32_t item, uint32_t* list,
		unsigned long long* len) {
	constexpr int kWarps = kThreads / 32;
	__shared__ uint32_t s_cnt[kWarps];
	__shared__ unsigned long long s_base;
	const uint32_t lane = threadIdx.x & 31u, wid = threadIdx.x >> 5;
	const unsigned m = __ballot_sync(0xffffffffu, take);
	if (lane == 0) s_cnt[wid] = __popc(m);
	__syncthreads();
	if (threadIdx.x == 0) {
		uint32_t tot = 0;
		for (int w = 0; w < kWarps; w++) {
			const uint32_t x = s_cnt[w];
			s_cnt[w] = tot;
			tot += x;
		}
		s_base = tot ? atomicAdd(len, (unsigned long long)tot) : 0ull;
	}
	__syncthreads();
	if (take) list[s_base + s_cnt[wid] + __popc(m & ((1u << lane) - 1u))] = item;
}

} // namespace lg

#endif // LG_QUEUE_CUH_
