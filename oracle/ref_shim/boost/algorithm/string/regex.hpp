// Stand-in for boost::algorithm::split_regex: the pieces of `s` between
// matches of `re`, in order, empty pieces included.  Test infrastructure for
// the reference-source oracle build.
#pragma once
#include <regex>
#include <string>
#include <vector>

namespace boost {
namespace algorithm {

inline std::vector<std::string>& split_regex(std::vector<std::string>& out, const std::string& s, const std::regex& re) {
  out.clear();
  std::sregex_token_iterator it(s.begin(), s.end(), re, -1), end;
  for (; it != end; ++it) out.push_back(*it);
  if (out.empty()) out.push_back(std::string());
  return out;
}

}  // namespace algorithm
using algorithm::split_regex;
}  // namespace boost
