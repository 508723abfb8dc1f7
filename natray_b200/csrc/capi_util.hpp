#pragma once
#include <string>

#include "natray.h"

namespace ntr {
// Records the message for ntr_last_error() and returns the status.
ntr_status fail(ntr_status s, const std::string& msg);
void clear_error();
}  // namespace ntr
