// The calling thread's last error message (returned by tdbem_last_error),
// for host code outside capi.cu.
#pragma once

#include <string>

namespace tdbem {
void set_last_error(const std::string& message);
}
