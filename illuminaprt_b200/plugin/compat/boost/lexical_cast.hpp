#pragma once
#include <sstream>
#include <string>
namespace boost { template <class T, class S> T lexical_cast(const S &s) { std::stringstream ss; ss << s; T t; ss >> t; return t; } }
