// Shared helpers of the hlrc library: per-thread error message and status
// plumbing used by both the host construction and the device entry points.
#pragma once

#include <cstdarg>
#include <cstdio>
#include <string>

#include "hlrc.h"

namespace hlrc {

// Records a printf-style message as the calling thread's last error and
// returns `st`, so call sites read `return fail(HLRC_ERR_ARG, "...")`.
hlrc_status fail(hlrc_status st, const char* fmt, ...)
#if defined(__GNUC__)
    __attribute__((format(printf, 2, 3)))
#endif
    ;

void clear_error();

}  // namespace hlrc
