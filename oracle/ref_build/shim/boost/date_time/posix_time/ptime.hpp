// Minimal boost::posix_time stand-in: microsecond-resolution instants and durations,
// the only operations the reference's sar/ sources use (+, -, microseconds(),
// total_microseconds()).
#pragma once

#include <cstdint>

namespace boost {
namespace posix_time {

struct time_duration {
    int64_t us = 0;
    int64_t total_microseconds() const { return us; }
};

struct ptime {
    int64_t us = 0;
};

inline time_duration microseconds(int64_t v) { return time_duration{v}; }
inline ptime operator+(ptime t, time_duration d) { return ptime{t.us + d.us}; }
inline ptime operator-(ptime t, time_duration d) { return ptime{t.us - d.us}; }
inline time_duration operator-(ptime a, ptime b) { return time_duration{a.us - b.us}; }

}  // namespace posix_time
}  // namespace boost
