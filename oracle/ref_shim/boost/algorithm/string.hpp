// Stand-in for the Boost string algorithms the SAMoS hot-path sources call:
// trim, to_lower, to_lower_copy.  Test infrastructure for the
// reference-source oracle build.
#pragma once
#include <algorithm>
#include <cctype>
#include <string>

namespace boost {
namespace algorithm {

inline void trim(std::string& s) {
  std::size_t b = 0, e = s.size();
  while (b < e && std::isspace((unsigned char)s[b])) ++b;
  while (e > b && std::isspace((unsigned char)s[e - 1])) --e;
  s = s.substr(b, e - b);
}
inline void to_lower(std::string& s) {
  std::transform(s.begin(), s.end(), s.begin(), [](unsigned char c) { return (char)std::tolower(c); });
}
inline std::string to_lower_copy(std::string s) {
  to_lower(s);
  return s;
}

}  // namespace algorithm
using algorithm::to_lower;
using algorithm::to_lower_copy;
using algorithm::trim;
}  // namespace boost
