#include "errors.hpp"

namespace blest {

static thread_local std::string g_last_error;

void set_last_error(const std::string& msg) { g_last_error = msg; }

}  // namespace blest

extern "C" const char* blest_last_error(void) { return blest::g_last_error.c_str(); }
