// Stand-in for SAMoS's src/parser/parse_parameters.hpp.  The plugin headers
// include it only for the parameter-map type; the Spirit grammar it also
// defines is not needed because the oracle driver hands each constructor a
// ready map.  Test infrastructure for the reference-source oracle build.
#ifndef __PARSE_PARAMETERS__
#define __PARSE_PARAMETERS__
#include <map>
#include <string>
typedef std::map<std::string, std::string> pairs_type;
#endif
