// Error plumbing and the version entry point of the C-ABI.
#include "common.cuh"

namespace ama {
static thread_local std::string g_last_error;
void set_error(const std::string& msg) { g_last_error = msg; }
}  // namespace ama

extern "C" const char* ama_last_error(void) { return ama::g_last_error.c_str(); }
extern "C" int ama_version(void) { return 100; }
