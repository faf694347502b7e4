// tpsc_host.h -- host-side helpers shared by the library's C++ files.
#pragma once
#include <string>

namespace tpsc {
// sets the message tpsc_last_error(NULL) returns; returns code
int static_fail(int code, const std::string &msg);
}  // namespace tpsc
