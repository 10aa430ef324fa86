// Error plumbing and the version entry point of the C-ABI.
#include "common.cuh"

namespace ama {
static thread_local std::string g_last_error;
void set_error(const std::string& msg) { g_last_error = msg; }
static std::atomic<uint64_t> g_memory_epoch{1};
uint64_t memory_epoch() { return g_memory_epoch.load(std::memory_order_acquire); }
void bump_memory_epoch() { g_memory_epoch.fetch_add(1, std::memory_order_acq_rel); }
}  // namespace ama

extern "C" const char* ama_last_error(void) { return ama::g_last_error.c_str(); }
extern "C" int ama_version(void) { return 100; }
