// Error channel of the C ABI: the message of the last failing call, per calling thread (ws_last_error).
#pragma once
#include <string>

namespace wsb {
void set_error(const std::string &msg);
const std::string &last_error();
inline int fail(int code, const std::string &msg) { set_error(msg); return code; }
}  // namespace wsb
