// Internal helpers shared by the host-side translation units of libcgc.
#pragma once
#include <cstdint>
#include <string>

#include "cgc.h"

namespace cgc {

// Records `msg` as the calling thread's last error and returns `code`.
int fail(int code, const std::string& msg);
// Clears the calling thread's last error and returns CGC_OK.
int ok();

}  // namespace cgc
