// sfp_internal.h -- helpers shared by the translation units of libsfp.so
// (not part of the C-ABI).
#pragma once
#include <string>

// record `msg` as the calling thread's last error (sfp_last_error) and return `code`
int sfp_set_error(int code, const std::string& msg);
