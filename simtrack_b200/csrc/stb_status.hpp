// Status codes shared by the C++ API and the C ABI: the STB_* values of
// include/simtrack_b200.h.
#pragma once
#include <string>

#include "simtrack_b200.h"

namespace stb {

// Thread-local message of the last failed call made on this thread.
void set_last_error(const std::string &msg);
const char *last_error();

}  // namespace stb
