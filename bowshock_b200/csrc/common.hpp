// Error reporting shared by every C entry point: a status code plus a
// thread-local message returned by bs_last_error().
#pragma once

#include <string>

#include "bowshock.h"

namespace bs {

void set_error(const std::string& message);
inline bs_status fail(bs_status status, const std::string& message) {
  set_error(message);
  return status;
}
inline bs_status ok() { return BS_OK; }

}  // namespace bs
