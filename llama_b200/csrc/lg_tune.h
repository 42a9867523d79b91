// lg_tune.h - launch parameters read by the kernels' host code.
#ifndef LG_TUNE_H_
#define LG_TUNE_H_

#include <stdint.h>

namespace lg {

// The current value of tunable `key` (LG_TUNE_*) for `device`.
int64_t tune_value(int device, int key);

} // namespace lg

#endif // LG_TUNE_H_
