// Stand-in for boost::regex: the standard library's ECMAScript regex, which
// accepts the one pattern the SAMoS particle reader uses ("\\s+|,|\\t").
// Test infrastructure for the reference-source oracle build.
#pragma once
#include <regex>
namespace boost {
using regex = std::regex;
}
