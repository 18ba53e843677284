// Status codes and the thread-local last-error message shared by every
// translation unit of libcvfes_b200.
#pragma once

#include <cstdarg>
#include <cstdio>
#include <string>

#include "cvfes_b200.h"

namespace cvfes {

std::string& last_error();

inline int fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    last_error() = buf;
    return code;
}

}  // namespace cvfes
