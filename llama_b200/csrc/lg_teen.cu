// lg_teen.cu - task "avg_teen_cnt" over a snapshot's in-CSR.
//
// Reference: ll_b_avg_teen_cnt::run (benchmark/benchmarks/avg_teen_cnt.h:
// 96-139): for every vertex n, teen_cnt[n] = number of in-neighbours t with
// 10 <= age[t] < 20 (age: the node property "age"); over the vertices with
// age[n] > K it sums the counts and returns (float)(sum / count).
//
// The ages become a bitset (teen_bits, one ballot per 32 vertices), the
// in-CSR is read flat (the snapshot's lg_snapshot_flatten CSR, or one built
// for the call), and one warp per 256-edge tile counts teen in-neighbours:
// lane j takes 8 consecutive edges (one 32-byte id load) and the matching
// byte of head bits, counts per row segment and adds each non-zero count to
// the row's total with one integer atomic (exact, so the order does not
// matter).  A second pass reduces over the vertices with age > K.
#include "lg_flat.cuh"

namespace lg {

constexpr int kTeenWarps = 8;

__global__ void teen_bits(const int32_t* age, uint64_t V, uint32_t* bits) {
	const uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	bool t = false;
	if (v < V) { const int32_t a = age[v]; t = a >= 10 && a < 20; }
	const unsigned m = __ballot_sync(0xffffffffu, t);
	if ((threadIdx.x & 31u) == 0 && v < V) bits[v >> 5] = m;
}

__global__ void __launch_bounds__(kTeenWarps * 32)
teen_tiles(const uint32_t* ids, const uint32_t* heads, const uint32_t* nz_rows,
		const uint32_t* tile_seg, uint32_t E, uint32_t ntiles, const uint32_t* bits,
		int32_t* teen_cnt) {
	const uint32_t lane = threadIdx.x & 31u;
	const uint32_t t = blockIdx.x * kTeenWarps + (threadIdx.x >> 5);
	if (t >= ntiles) return;
	const uint32_t eb = t * kFlatTile + lane * kFlatPerLane;
	const uint32_t hb = __ldg(reinterpret_cast<const unsigned char*>(heads)
			+ (size_t)t * (kFlatTile / 8) + lane);
	uint32_t id[kFlatPerLane];
	if (eb + kFlatPerLane <= E) {
		asm("ld.global.cs.v8.u32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
			: "=r"(id[0]), "=r"(id[1]), "=r"(id[2]), "=r"(id[3]),
			  "=r"(id[4]), "=r"(id[5]), "=r"(id[6]), "=r"(id[7])
			: "l"(ids + eb));
	} else {
#pragma unroll
		for (int i = 0; i < kFlatPerLane; i++) id[i] = eb + i < E ? __ldcs(ids + eb + i) : kNoId;
	}
	uint32_t teen = 0;
#pragma unroll
	for (int i = 0; i < kFlatPerLane; i++)
		if (id[i] != kNoId) teen |= ((__ldg(bits + (id[i] >> 5)) >> (id[i] & 31u)) & 1u) << i;
	// heads in the lanes to the left
	uint32_t before = __popc(hb);
#pragma unroll
	for (int o = 1; o < 32; o <<= 1) {
		const uint32_t q = __shfl_up_sync(0xffffffffu, before, o);
		if (lane >= (uint32_t)o) before += q;
	}
	before -= __popc(hb);
	// the row of this lane's first edge is the last one begun at or before it
	uint32_t row = __ldg(tile_seg + t) + before - 1u;
	int32_t c = 0;
#pragma unroll
	for (int i = 0; i < kFlatPerLane; i++) {
		if ((hb >> i) & 1u) {
			if (c) atomicAdd(teen_cnt + __ldg(nz_rows + row), c);
			row++;
			c = 0;
		}
		c += (teen >> i) & 1u;
	}
	if (c) atomicAdd(teen_cnt + __ldg(nz_rows + row), c);
}

// sums[0] += teen_cnt over vertices with age > K, sums[1] += their number.
__global__ void teen_reduce(const int32_t* age, const int32_t* teen_cnt, uint64_t V, int K,
		unsigned long long* sums) {
	unsigned long long s = 0, c = 0;
	for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < V;
			v += (uint64_t)gridDim.x * blockDim.x) {
		if (age[v] > K) { s += (unsigned long long)(long long)teen_cnt[v]; c++; }
	}
#pragma unroll
	for (int o = 16; o > 0; o >>= 1) {
		s += __shfl_xor_sync(0xffffffffu, s, o);
		c += __shfl_xor_sync(0xffffffffu, c, o);
	}
	if ((threadIdx.x & 31u) == 0) {
		if (s) atomicAdd(sums, s);
		if (c) atomicAdd(sums + 1, c);
	}
}

} // namespace lg

using namespace lg;

extern "C" lg_status lg_avg_teen_cnt(lg_snapshot* sn, const int32_t* age, int K,
		int32_t* teen_cnt, lg_teen_result* result) {
	clear_error();
	if (!sn || !age) return set_error(LG_EINVAL, "null argument");
	if (!sn->in.present)
		return set_error(LG_ESTATE, "avg_teen_cnt needs the in-CSR (reverse edges)");
	lg_store* s = sn->store;
	LG_CUDA(cudaSetDevice(s->device), "cudaSetDevice");
	cudaStream_t st = s->stream;
	const uint64_t V = sn->V;
	const unsigned B = 256;
	DevBuf* sc = s->scratch;

	const int32_t* d_age = age;
	if (!is_device_pointer(age)) {
		LG_TRY(sc[0].reserve(std::max<uint64_t>(V, 1) * sizeof(int32_t)));
		LG_CUDA(cudaMemcpyAsync(sc[0].p, age, V * sizeof(int32_t), cudaMemcpyHostToDevice, st),
				"age upload");
		s->h2d_bytes += V * sizeof(int32_t);
		d_age = sc[0].as<int32_t>();
	}
	const bool dev_out = teen_cnt && is_device_pointer(teen_cnt);
	int32_t* cnt = teen_cnt;
	if (!dev_out) {
		LG_TRY(sc[1].reserve(std::max<uint64_t>(V, 1) * sizeof(int32_t)));
		cnt = sc[1].as<int32_t>();
	}
	LG_TRY(sc[2].reserve(((V + 31) / 32 + 1) * sizeof(uint32_t)));
	LG_TRY(sc[3].reserve(2 * sizeof(unsigned long long)));
	uint32_t* bits = sc[2].as<uint32_t>();
	unsigned long long* sums = sc[3].as<unsigned long long>();

	const FlatCsr* f = sn->flat[1];
	if (!f) {
		if (!s->flat_scratch) s->flat_scratch = new FlatCsr;
		LG_TRY(build_flat(sn, 1, *s->flat_scratch, false));
		f = s->flat_scratch;
	}
	LG_CUDA(cudaMemsetAsync(cnt, 0, V * sizeof(int32_t), st), "clear counts");
	LG_CUDA(cudaMemsetAsync(sums, 0, 2 * sizeof(unsigned long long), st), "clear sums");
	teen_bits<<<grid_for(V, B), B, 0, st>>>(d_age, V, bits);
	if (f->ntiles > 0)
		teen_tiles<<<(f->ntiles + kTeenWarps - 1) / kTeenWarps, kTeenWarps * 32, 0, st>>>(
				f->ids.as<uint32_t>(), f->heads(), f->nz_rows(), f->tile_seg(), (uint32_t)f->E,
				f->ntiles, bits, cnt);
	teen_reduce<<<592, B, 0, st>>>(d_age, cnt, V, K, sums);
	LG_CUDA(cudaGetLastError(), "avg_teen_cnt");
	s->launches += 2 + (f->ntiles > 0);
	unsigned long long h[2] = {0, 0};
	LG_CUDA(cudaMemcpyAsync(h, sums, sizeof(h), cudaMemcpyDeviceToHost, st), "d2h");
	s->d2h_bytes += sizeof(h);
	if (teen_cnt && !dev_out) LG_TRY(copy_out(s, teen_cnt, cnt, V * sizeof(int32_t)));
	LG_CUDA(cudaStreamSynchronize(st), "avg_teen_cnt");
	if (result) {
		result->teen_sum = (int64_t)h[0];
		result->vertices = (int64_t)h[1];
		const double avg = h[1] == 0 ? 0.0 : (double)(int64_t)h[0] / (double)h[1];
		result->average = (double)(float)avg;
	}
	return LG_OK;
}
