// Thread-local error message and version of the library.
#include "../common.hpp"

namespace {
thread_local std::string g_last_error;
}

namespace bs {
void set_error(const std::string& message) { g_last_error = message; }
}  // namespace bs

extern "C" {
const char* bs_last_error(void) { return g_last_error.c_str(); }
const char* bs_version(void) { return "bowshock_b200 0.1 (sm_100a)"; }
}
