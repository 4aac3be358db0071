// Stand-in for boost::lexical_cast as the SAMoS hot-path sources use it:
// text -> number (the whole text must be consumed, else bad_lexical_cast)
// and number -> text.  Doubles parse with strtod, which rounds correctly, so
// a value written with 17 significant digits reads back bit for bit.
// Test infrastructure for the reference-source oracle build.
#pragma once
#include <cctype>
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <sstream>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <typeinfo>

namespace boost {

class bad_lexical_cast : public std::bad_cast {
 public:
  const char* what() const noexcept override { return "bad lexical cast"; }
};

namespace shim_detail {
inline std::string to_text(const std::string& s) { return s; }
inline std::string to_text(const char* s) { return s; }
inline std::string to_text(char c) { return std::string(1, c); }
inline std::string to_text(bool b) { return b ? "1" : "0"; }
template <class T>
std::string to_text(const T& v) {
  if constexpr (std::is_floating_point<T>::value) {
    char buf[64];
    std::snprintf(buf, sizeof buf, "%.17g", (double)v);
    return buf;
  } else {
    std::ostringstream os;
    os << v;
    return os.str();
  }
}
}  // namespace shim_detail

template <class T, class S>
T lexical_cast(const S& src) {
  if constexpr (std::is_same<T, std::string>::value) {
    return shim_detail::to_text(src);
  } else {
    std::string s = shim_detail::to_text(src);
    if (s.empty()) throw bad_lexical_cast();
    const char* b = s.c_str();
    char* e = nullptr;
    errno = 0;
    if constexpr (std::is_floating_point<T>::value) {
      double v = std::strtod(b, &e);
      if (e == b || *e != '\0' || std::isspace((unsigned char)s[0])) throw bad_lexical_cast();
      return static_cast<T>(v);
    } else if constexpr (std::is_same<T, bool>::value) {
      if (s == "1") return true;
      if (s == "0") return false;
      throw bad_lexical_cast();
    } else if constexpr (std::is_integral<T>::value) {
      long long v = std::strtoll(b, &e, 10);
      if (e == b || *e != '\0' || errno == ERANGE || std::isspace((unsigned char)s[0])) throw bad_lexical_cast();
      if (std::is_unsigned<T>::value && v < 0) throw bad_lexical_cast();
      return static_cast<T>(v);
    } else {
      std::istringstream is(s);
      T v;
      is >> v;
      if (is.fail() || !is.eof()) throw bad_lexical_cast();
      return v;
    }
  }
}

}  // namespace boost
