// fmt shim for the reference's log messages (the messages are discarded).
#pragma once

#include <string>

namespace fmt {
template <class... A>
std::string format(const char* f, A&&...) {
    return f;
}
}  // namespace fmt
