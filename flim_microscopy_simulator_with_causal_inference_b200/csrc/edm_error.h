// edm_error.h — the library's last-error slot (read by edm_last_error()).
#pragma once
#include <string>

namespace edm {
// Records msg as this thread's last error and returns code.
int report_error(int code, const std::string& msg);
}  // namespace edm
