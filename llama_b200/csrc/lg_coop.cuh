// lg_coop.cuh - building blocks of the one-launch traversals (lg_bfs_levels.cu,
// lg_sssp_levels.cu): a grid barrier for cooperative launches whose waits
// are bounded by the global timer, and CTA-wide sums and scans.
#ifndef LG_COOP_CUH_
#define LG_COOP_CUH_

#include <cuda_runtime.h>
#include <stdint.h>

namespace lg {

// Barrier state in device memory; count must be 0 before the launch.
struct CoopBar {
	unsigned int count;
	unsigned int gen;
	unsigned int err;      // bit 0: a barrier wait ran out; higher bits: the caller's
	unsigned int pad;
};

constexpr uint64_t kCoopWaitNs = 1000000000ull;   // a barrier wait gives up after 1 s

__device__ __forceinline__ uint64_t global_ns() {
	uint64_t t;
	asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
	return t;
}

// Barrier over all CTAs of a cooperative grid (all co-resident).  Thread 0
// of each CTA publishes the CTA's writes (fence), arrives, and waits for the
// generation to move on; false once any CTA gave up waiting or set an error.
__device__ inline bool grid_barrier(CoopBar* b) {
	__shared__ int s_ok;
	__syncthreads();
	if (threadIdx.x == 0) {
		int ok = 1;
		volatile unsigned int* gen = &b->gen;
		const unsigned int g = *gen;
		__threadfence();
		if (atomicAdd(&b->count, 1u) == gridDim.x - 1u) {
			atomicExch(&b->count, 0u);
			__threadfence();
			atomicAdd(&b->gen, 1u);
		} else {
			const uint64_t t0 = global_ns();
			volatile unsigned int* err = &b->err;
			while (*gen == g) {
				if (*err) {                  // a CTA left on an error: it will not arrive
					ok = 0;
					break;
				}
				if (global_ns() - t0 > kCoopWaitNs) {
					atomicOr(&b->err, 1u);
					ok = 0;
					break;
				}
				__nanosleep(64);
			}
		}
		__threadfence();
		if (*(volatile unsigned int*)&b->err) ok = 0;
		s_ok = ok;
	}
	__syncthreads();
	return s_ok != 0;
}

// Sum of x over a CTA of kWarps warps, returned to every thread (all
// threads call it).
template <int kWarps>
__device__ __forceinline__ unsigned long long block_sum(unsigned long long x) {
	__shared__ unsigned long long s_part[kWarps];
	const uint32_t lane = threadIdx.x & 31u, wid = threadIdx.x >> 5;
#pragma unroll
	for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
	__syncthreads();                     // s_part free from a previous call
	if (lane == 0) s_part[wid] = x;
	__syncthreads();
	unsigned long long t = 0;
#pragma unroll
	for (int w = 0; w < kWarps; w++) t += s_part[w];
	return t;
}

// Exclusive scan of x over a CTA of kWarps warps in thread order; *total =
// the CTA's sum (all threads call it).
template <int kWarps>
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t x, uint32_t* total) {
	__shared__ uint32_t s_warp[kWarps];
	const uint32_t lane = threadIdx.x & 31u, wid = threadIdx.x >> 5;
	uint32_t inc = x;
#pragma unroll
	for (int o = 1; o < 32; o <<= 1) {
		const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
		if (lane >= (uint32_t)o) inc += y;
	}
	__syncthreads();
	if (lane == 31u) s_warp[wid] = inc;
	__syncthreads();
	uint32_t before = 0, all = 0;
#pragma unroll
	for (int w = 0; w < kWarps; w++) {
		const uint32_t s = s_warp[w];
		if (w < (int)wid) before += s;
		all += s;
	}
	*total = all;
	return before + inc - x;
}

// Co-resident CTAs of `kernel` at `threads` per CTA on `device` (SMs x CTAs
// per SM), 0 when the device has no cooperative launch.
inline int coop_grid_size(const void* kernel, int threads, int device) {
	int coop = 0, sms = 0, per_sm = 0;
	if (cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device) != cudaSuccess ||
			cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess ||
			cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, 0) !=
					cudaSuccess) {
		cudaGetLastError();
		return 0;
	}
	return coop && sms > 0 && per_sm > 0 ? sms * per_sm : 0;
}

} // namespace lg

#endif // LG_COOP_CUH_
