// Stand-in: the writers live in ptree.hpp (oracle build test infrastructure).
#pragma once
#include "ptree.hpp"
