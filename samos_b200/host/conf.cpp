// conf.cpp -- the conf-file line syntax of the reference: one command per
// line, `#` comments, and `{ key = value; flag; ... }` parameter blocks
// (key_value_sequence, src/parser/parse_parameters.hpp:45-52: keys
// [a-zA-Z_][a-zA-Z_0-9]*, values [-a-zA-Z_0-9+./]+, separators ';' or ',').
#include <cctype>

#include "samos_host.hpp"

namespace samos_host {

std::string trim(const std::string& s) {
  size_t a = 0, b = s.size();
  while (a < b && std::isspace((unsigned char)s[a])) a++;
  while (b > a && std::isspace((unsigned char)s[b - 1])) b--;
  return s.substr(a, b - a);
}

namespace {

struct Cursor {
  const std::string& s;
  size_t i = 0;
  void skip() { while (i < s.size() && std::isspace((unsigned char)s[i])) i++; }
  bool eat(char c) { skip(); if (i < s.size() && s[i] == c) { i++; return true; } return false; }
  bool at_end() { skip(); return i >= s.size(); }
};

bool key_char(char c, bool first) {
  return std::isalpha((unsigned char)c) || c == '_' || (!first && std::isdigit((unsigned char)c));
}
bool value_char(char c) {
  return std::isalnum((unsigned char)c) || c == '-' || c == '_' || c == '+' || c == '.' || c == '/';
}

bool parse_pair(Cursor& c, Params& out) {
  c.skip();
  size_t a = c.i;
  if (a >= c.s.size() || !key_char(c.s[a], true)) return false;
  while (c.i < c.s.size() && key_char(c.s[c.i], false)) c.i++;
  const std::string key = c.s.substr(a, c.i - a);
  std::string value;
  if (c.eat('=')) {
    c.skip();
    size_t b = c.i;
    while (c.i < c.s.size() && value_char(c.s[c.i])) c.i++;
    if (c.i == b) return false;
    value = c.s.substr(b, c.i - b);
  }
  // std::map insertion of a fusion pair keeps the first occurrence
  out.emplace(key, value);
  return true;
}

}  // namespace

bool parse_params(const std::string& text, Params& out) {
  out.clear();
  Cursor c{text};
  if (!c.eat('{')) return false;
  if (c.eat('}')) return c.at_end();
  if (!parse_pair(c, out)) return false;
  for (;;) {
    const size_t save = c.i;
    if (c.eat(';') || c.eat(',')) {
      if (parse_pair(c, out)) continue;
      c.i = save;
    }
    break;
  }
  while (c.eat(';')) {
  }
  if (!c.eat('}')) return false;
  return c.at_end();
}

void split_command(const std::string& line, std::string& cmd, std::string& rest) {
  const std::string t = trim(line);
  size_t i = 0;
  while (i < t.size() && !std::isspace((unsigned char)t[i]) && t[i] != '{') i++;
  cmd = t.substr(0, i);
  rest = trim(t.substr(i));
}

bool split_type_params(const std::string& rest, std::string& type, std::string& params, bool file_name) {
  const std::string t = trim(rest);
  size_t i = 0;
  // log / dump names are file names: letters, digits, '_' and '.' (parse_log_dump.hpp:63)
  while (i < t.size() && (std::isalnum((unsigned char)t[i]) || t[i] == '_' || (file_name && t[i] == '.'))) i++;
  type = t.substr(0, i);
  params = trim(t.substr(i));
  if (params.empty()) params = "{}";
  return !type.empty();
}

}  // namespace samos_host
