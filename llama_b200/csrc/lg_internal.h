// lg_internal.h - error reporting shared by the host and device translation
// units of liblg.
#ifndef LG_INTERNAL_H_
#define LG_INTERNAL_H_

#include "../../include/lg.h"

namespace lg {

// Record `msg` as the calling thread's last error and return `st`.
lg_status set_error(lg_status st, const char* fmt, ...)
#if defined(__GNUC__)
	__attribute__((format(printf, 2, 3)))
#endif
	;
void clear_error();

} // namespace lg

#endif // LG_INTERNAL_H_
