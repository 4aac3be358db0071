// Stand-in for boost::property_tree as SAMoS's Messenger uses it: a
// key -> value store for its optional run-configuration record.  Writing the
// record is a no-op here (the oracle build never asks for one).  Test
// infrastructure for the reference-source oracle build.
#pragma once
#include <map>
#include <string>
#include <utility>
#include <vector>

namespace boost {
namespace property_tree {

class ptree {
 public:
  void put(const std::string& k, const std::string& v) {
    for (auto& kv : items_)
      if (kv.first == k) { kv.second = v; return; }
    items_.emplace_back(k, v);
  }
  void add(const std::string& k, const std::string& v) { items_.emplace_back(k, v); }

 private:
  std::vector<std::pair<std::string, std::string>> items_;
};

inline void write_json(const std::string&, const ptree&) {}
inline void write_xml(const std::string&, const ptree&) {}
inline void write_info(const std::string&, const ptree&) {}

}  // namespace property_tree
}  // namespace boost
