// Logging shim for compiling the reference's sar/ sources without Boost.Log:
// LOGV..LOGE become streams that discard everything.
#pragma once

#include <ostream>

namespace refshim {
struct NullLog {
    template <class T>
    NullLog& operator<<(const T&) {
        return *this;
    }
    NullLog& operator<<(std::ostream& (*)(std::ostream&)) { return *this; }
};
}  // namespace refshim

#define LOGV refshim::NullLog{}
#define LOGD refshim::NullLog{}
#define LOGI refshim::NullLog{}
#define LOGW refshim::NullLog{}
#define LOGE refshim::NullLog{}
