// Stand-in for the boost string algorithms the engine's scene loaders use.
#pragma once
#include <cctype>
#include <string>

namespace boost {
inline void trim(std::string &s)
{
    size_t b = 0, e = s.size();
    while (b < e && std::isspace((unsigned char)s[b])) b++;
    while (e > b && std::isspace((unsigned char)s[e - 1])) e--;
    s = s.substr(b, e - b);
}
inline std::string to_upper_copy(const std::string &s)
{
    std::string r(s);
    for (size_t i = 0; i < r.size(); i++) r[i] = (char)std::toupper((unsigned char)r[i]);
    return r;
}
inline std::string to_lower_copy(const std::string &s)
{
    std::string r(s);
    for (size_t i = 0; i < r.size(); i++) r[i] = (char)std::tolower((unsigned char)r[i]);
    return r;
}
inline void to_upper(std::string &s) { s = to_upper_copy(s); }
inline void to_lower(std::string &s) { s = to_lower_copy(s); }
}  // namespace boost
