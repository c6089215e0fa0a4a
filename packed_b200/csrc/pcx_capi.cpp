// C ABI plumbing: per-thread error messages and the version string.
#include "pcx_host.hpp"

namespace {
thread_local std::string g_last_error;
}

int pcx_fail(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}

extern "C" const char* pcx_last_error(void) { return g_last_error.c_str(); }

extern "C" const char* pcx_version(void) { return "packed-b200 0.1.0 (sm_100a)"; }
