// Thread-local last-error text and the status helper shared by the C ABI functions.
#pragma once

#include <string>

namespace ddm {

// Records `message` as this thread's last error and returns `status`.
int fail(int status, const std::string &message);
void clear_error();
const char *last_error();

}  // namespace ddm
