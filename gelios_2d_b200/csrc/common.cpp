// Error reporting shared by the C ABI of gelios_b200.
#include <string>

#include "../../include/gelios_b200.h"

namespace gelios {
namespace {
thread_local std::string g_last_error;
}
void set_error(const std::string& msg) { g_last_error = msg; }
}  // namespace gelios

extern "C" const char* gelios_last_error(void) { return gelios::g_last_error.c_str(); }
extern "C" int gelios_abi_version(void) { return GELIOS_ABI_VERSION; }
