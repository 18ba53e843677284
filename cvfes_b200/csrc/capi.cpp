// Library-wide C-ABI entry points: last error message and version.
#include <string>

#include "cvfes_b200.h"
#include "errors.h"

std::string& cvfes::last_error() {
    thread_local std::string msg;
    return msg;
}

extern "C" const char* cvfes_last_error(void) { return cvfes::last_error().c_str(); }

extern "C" int cvfes_version(void) { return 100; }
