#pragma once

#include <exception>
#include <new>
#include <string>

#include "b2r.h"

namespace b2r {

void set_error(std::string msg);

inline int fail(int status, std::string msg) {
  set_error(std::move(msg));
  return status;
}

}  // namespace b2r

// No exception may cross the C ABI: every entry point body runs inside this
// guard and maps exceptions onto status codes.
#define B2R_API_GUARD(...)                                              \
  try {                                                                  \
    __VA_ARGS__                                                          \
  } catch (std::bad_alloc const&) {                                      \
    return b2r::fail(B2R_ERR_OUT_OF_MEMORY, "host allocation failed");   \
  } catch (std::exception const& e) {                                    \
    return b2r::fail(B2R_ERR_INTERNAL, e.what());                        \
  } catch (...) {                                                        \
    return b2r::fail(B2R_ERR_INTERNAL, "unknown exception");             \
  }
