// TEST INFRASTRUCTURE: the boost posix_time subset the reference's timing
// utilities use (src/Utilities/timingUtilities.hh), on std::chrono.
#ifndef ORACLE_REFSHIM_BOOST_POSIX_TIME
#define ORACLE_REFSHIM_BOOST_POSIX_TIME
#include <chrono>
namespace boost {
namespace posix_time {
struct time_duration {
  long long ns;
  long long total_nanoseconds() const { return ns; }
};
struct ptime {
  std::chrono::steady_clock::time_point t;
  time_duration operator-(const ptime& o) const {
    return time_duration{(long long)std::chrono::duration_cast<std::chrono::nanoseconds>(t - o.t).count()};
  }
};
struct microsec_clock {
  static ptime local_time() { return ptime{std::chrono::steady_clock::now()}; }
};
}
}
#endif
