// Error reporting shared by the host translation units of libakb.
#pragma once

#include <string>

namespace akb {
// records msg as the thread's last error and returns code
int fail(int code, const std::string &msg);
}  // namespace akb
