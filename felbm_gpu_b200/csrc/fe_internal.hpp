// Internal helpers shared by the host translation units: the thread-local
// last-error message behind fe_last_error(), and status helpers.
#pragma once
#include <string>

namespace fe {

// Record a failure for fe_last_error() and return its status code.
int fe_fail(int status, const std::string& msg);
void fe_clear_error();

}  // namespace fe

using fe::fe_fail;
