// Stand-in for the part of boost::filesystem::path the engine's scene loaders
// use to split a file name from its directory ('/'-separated paths).
#pragma once
#include <string>

namespace boost {
namespace filesystem {
class path {
public:
    path() {}
    path(const std::string &s) : s_(s) {}
    path(const char *s) : s_(s) {}
    path filename() const
    {
        const size_t k = s_.find_last_of('/');
        return path(k == std::string::npos ? s_ : s_.substr(k + 1));
    }
    path parent_path() const
    {
        const size_t k = s_.find_last_of('/');
        return path(k == std::string::npos ? std::string() : s_.substr(0, k));
    }
    path operator/(const std::string &r) const { return path(s_.empty() ? r : s_ + "/" + r); }
    path operator/(const path &r) const { return *this / r.s_; }
    std::string string() const { return s_; }

private:
    std::string s_;
};
}  // namespace filesystem
}  // namespace boost
