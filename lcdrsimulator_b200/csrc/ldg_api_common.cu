// Error recording and version string of the C ABI.
#include <string>

#include "ldg_api_common.h"

namespace ldg {
namespace {
thread_local std::string g_last_error;
}
void set_error(const std::string& msg) { g_last_error = msg; }
void clear_error() { g_last_error.clear(); }
}  // namespace ldg

extern "C" {
const char* ldg_last_error(void) { return ldg::g_last_error.c_str(); }
const char* ldg_version(void) { return "ldg_b200 0.1 (sm_100a)"; }
}
