// Internal declarations shared by the library's translation units.
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>

#include "../../include/cgp_b200.h"

namespace cgp {

// ---------------------------------------------------------------- errors
// Thread-local last-error message; every C entry point returns a status and
// records the message here (no exception crosses the C boundary).
cgp_status set_error(cgp_status code, const std::string& msg);
void clear_error();

uint64_t mix64(uint64_t x);

// Largest mask width: 16 x 64-bit words = 1024 queries per traversal group.
constexpr int kMaxWords = 16;

}  // namespace cgp
