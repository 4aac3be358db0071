// Stand-in for the Boost.Date_Time piece SAMoS's Messenger uses: the local
// time stamped on each message.  Test infrastructure for the
// reference-source oracle build.
#pragma once
#include <ctime>
#include <ostream>

namespace boost {
namespace posix_time {

struct ptime {
  std::time_t t;
};
inline std::ostream& operator<<(std::ostream& os, const ptime& p) {
  char buf[64];
  std::tm tmv;
  localtime_r(&p.t, &tmv);
  std::strftime(buf, sizeof buf, "%Y-%b-%d %H:%M:%S", &tmv);
  return os << buf;
}
struct second_clock {
  static ptime local_time() { return ptime{std::time(nullptr)}; }
};

}  // namespace posix_time
namespace gregorian {}
}  // namespace boost
