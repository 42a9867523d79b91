// lg_sort.cuh - device sort and de-duplication helpers (lg_sort.cu).
#ifndef LG_SORT_CUH_
#define LG_SORT_CUH_

#include "lg_device.cuh"

namespace lg {

// Stable LSD radix sort of n 64-bit keys (and an optional u32 payload) on the
// store's stream.  The result ends up either in the input arrays or in the
// temporaries; *sorted_keys / *sorted_pay point at it.
lg_status radix_sort_u64(lg_store* s, unsigned long long* keys, uint32_t* payload,
		uint64_t n, DevBuf& tmp_keys, DevBuf& tmp_pay, DevBuf& counts, DevBuf& scan_tmp,
		unsigned long long** sorted_keys, uint32_t** sorted_pay);

// Copy the first of every run of equal keys (sorted input) to `out`; the
// number kept is returned in *n_out (this synchronises the stream).
lg_status unique_u64(lg_store* s, const unsigned long long* keys, uint64_t n,
		unsigned long long* out, DevBuf& flags, DevBuf& scan_tmp, uint64_t* n_out);

} // namespace lg

#endif // LG_SORT_CUH_
