// Per-thread last-error message of the hlrc C ABI.
#include "common.hpp"

#include <cstring>

namespace hlrc {

namespace {
thread_local char g_last_error[1024] = {0};
}

hlrc_status fail(hlrc_status st, const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
    va_end(ap);
    return st;
}

void clear_error() { g_last_error[0] = 0; }

}  // namespace hlrc

extern "C" const char* hlrc_last_error(void) { return hlrc::g_last_error; }

extern "C" int hlrc_abi_version(void) { return HLRC_ABI_VERSION; }

extern "C" void hlrc_default_options(hlrc_options* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->precision = HLRC_PREC_F64;
    o->max_nrhs = 1;
    o->mixed_eps = 1e-6;
    o->device = -1;
}
