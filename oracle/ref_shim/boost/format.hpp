// Stand-in for the part of Boost.Format that the SAMoS hot-path sources use:
// `format("... %d ...") % a % b`, streamed or turned into a string.  Each
// `%` argument fills the next printf-style directive.  Only message and dump
// text goes through it; no number that the parity tests compare does.
// Test infrastructure for the reference-source oracle build.
#pragma once
#include <algorithm>
#include <cstdio>
#include <ostream>
#include <sstream>
#include <string>
#include <type_traits>

namespace boost {

class format {
 public:
  explicit format(const std::string& f) : fmt_(f), pos_(0) { advance(); }
  explicit format(const char* f) : format(std::string(f)) {}

  template <class T>
  format& operator%(const T& v) {
    std::size_t start = pos_;
    if (start >= fmt_.size()) return *this;  // more arguments than directives
    std::size_t end = start + 1;
    while (end < fmt_.size() && std::string("diouxXeEfFgGcsp").find(fmt_[end]) == std::string::npos) ++end;
    std::string spec = fmt_.substr(start, end - start + 1);
    char conv = end < fmt_.size() ? fmt_[end] : 's';
    out_ += render(spec, conv, v);
    pos_ = end + 1;
    advance();
    return *this;
  }

  std::string str() const { return out_ + (pos_ < fmt_.size() ? fmt_.substr(pos_) : std::string()); }
  friend std::ostream& operator<<(std::ostream& os, const format& f) { return os << f.str(); }

 private:
  // copy literal text up to the next directive; "%%" is a literal percent
  void advance() {
    while (pos_ < fmt_.size()) {
      if (fmt_[pos_] == '%') {
        if (pos_ + 1 < fmt_.size() && fmt_[pos_ + 1] == '%') { out_ += '%'; pos_ += 2; continue; }
        return;
      }
      out_ += fmt_[pos_++];
    }
  }
  static std::string printf_spec(const std::string& spec, const char* len, char conv) {
    return spec.substr(0, spec.size() - 1) + len + conv;
  }
  template <class T>
  static std::string render(const std::string& spec, char conv, const T& v) {
    char buf[512];
    if constexpr (std::is_integral<T>::value) {
      if (conv == 'd' || conv == 'i' || conv == 'u' || conv == 'x' || conv == 'X' || conv == 'o' || conv == 'c') {
        std::snprintf(buf, sizeof buf, printf_spec(spec, "ll", conv == 'c' ? 'd' : conv).c_str(), (long long)v);
      } else {
        std::snprintf(buf, sizeof buf, spec.c_str(), (double)v);
      }
      return buf;
    } else if constexpr (std::is_floating_point<T>::value) {
      if (conv == 'd' || conv == 'i' || conv == 'u' || conv == 's') {
        std::ostringstream os;
        os << v;
        return os.str();
      }
      std::snprintf(buf, sizeof buf, spec.c_str(), (double)v);
      return buf;
    } else {
      std::ostringstream os;
      os << v;
      return os.str();
    }
  }

  std::string fmt_;
  std::size_t pos_;
  std::string out_;
};

}  // namespace boost
