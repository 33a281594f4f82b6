// errors.h -- thread-local last-error message shared by the C ABI entry points.
#pragma once
#include <string>

namespace dgtd {
// Record `msg` as the calling thread's last error and return `code`.
int set_error(int code, const std::string& msg);
}  // namespace dgtd
