// The library's per-thread last-error message (read through lbg_last_error).
#pragma once
#include <string>

namespace lbg {
void set_last_error(const std::string& msg);
}
