// Minimal boost::format stand-in: positional directives are replaced in order
// by the streamed arguments. Used only for ToString() text in the reference.
#pragma once
#include <string>
#include <sstream>
namespace boost {
class format {
  std::string fmt_; std::string out_; size_t pos_ = 0;
  void advance(const std::string &arg) {
    while (pos_ < fmt_.size()) {
      char c = fmt_[pos_];
      if (c == '%' && pos_ + 1 < fmt_.size() && fmt_[pos_ + 1] == '%') { out_ += '%'; pos_ += 2; continue; }
      if (c == '%') {
        size_t q = pos_ + 1;
        while (q < fmt_.size() && std::string("0123456789.-+ #lhL").find(fmt_[q]) != std::string::npos) q++;
        if (q < fmt_.size() && fmt_[q] == '%') q++;            // %1% style
        else if (q < fmt_.size()) q++;                          // %s / %d / %f style
        pos_ = q; out_ += arg; return;
      }
      out_ += c; pos_++;
    }
    out_ += arg;
  }
public:
  format() {}
  explicit format(const std::string &f) : fmt_(f) {}
  explicit format(const char *f) : fmt_(f) {}
  template <class T> format &operator%(const T &v) { std::ostringstream s; s << v; advance(s.str()); return *this; }
  std::string str() const { return out_ + fmt_.substr(pos_ < fmt_.size() ? pos_ : fmt_.size()); }
};
inline std::string str(const format &f) { return f.str(); }
template <class C, class T> std::basic_ostream<C, T> &operator<<(std::basic_ostream<C, T> &o, const format &f) { return o << f.str(); }
}
