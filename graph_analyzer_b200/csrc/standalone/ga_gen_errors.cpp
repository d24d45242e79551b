// ga_gen_errors.cpp - error reporting for libga_gen.so, the generators built without the rest of the library
// (libga_b200 has its own, in ga_host.cpp): fail() records the message that ga_last_error() returns.
#include <cstdarg>
#include <cstdio>
#include <string>

#include "ga_internal.h"

namespace ga {

static thread_local std::string t_err;

ga_status fail(ga_status s, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    t_err = buf;
    return s;
}

}  // namespace ga

extern "C" const char* ga_last_error(void) { return ga::t_err.c_str(); }
