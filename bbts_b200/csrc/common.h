// Shared host-side helpers of the bbts_b200 library.
#pragma once
#include <string>

namespace bbx {

// Records a formatted message as the calling thread's last error and returns `code`.
int set_error(int code, const char* fmt, ...);
const std::string& last_error();

}  // namespace bbx
