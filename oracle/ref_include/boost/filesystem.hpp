/*
 * Stands in for Boost.Filesystem when oracle/Makefile compiles the
 * reference's listmode sources (Boost is not installed here).  Paths are
 * plain strings; only the members those sources name exist.  The checked
 * code paths (LUT creation, rebinning, histogramming, the span-9 fold) take
 * no path argument: the harness opens the event file itself.  Test
 * infrastructure only.
 */
#pragma once
#include <fstream>  // the real header brings the file streams in (boost/filesystem/fstream.hpp)
#include <ostream>
#include <string>

namespace boost {
namespace filesystem {

class path {
 public:
  path() {}
  path(const char *s) : s_(s ? s : "") {}
  path(const std::string &s) : s_(s) {}
  const std::string &string() const { return s_; }
  const char *c_str() const { return s_.c_str(); }
  bool empty() const { return s_.empty(); }
  path filename() const { return path(s_.substr(s_.find_last_of('/') == std::string::npos ? 0 : s_.find_last_of('/') + 1)); }
  path parent_path() const {
    const size_t k = s_.find_last_of('/');
    return k == std::string::npos ? path() : path(s_.substr(0, k));
  }
  path extension() const {
    const std::string f = filename().string();
    const size_t k = f.find_last_of('.');
    return k == std::string::npos ? path() : path(f.substr(k));
  }
  path stem() const {
    const std::string f = filename().string();
    const size_t k = f.find_last_of('.');
    return path(k == std::string::npos ? f : f.substr(0, k));
  }
  path &replace_extension(const path &e = path()) {
    const std::string x = extension().string();
    if (!x.empty()) s_.resize(s_.size() - x.size());
    s_ += e.string();
    return *this;
  }
  path &operator/=(const path &p) {
    if (!s_.empty() && s_.back() != '/') s_ += '/';
    s_ += p.s_;
    return *this;
  }
  path &operator+=(const std::string &p) {
    s_ += p;
    return *this;
  }
  bool operator==(const path &o) const { return s_ == o.s_; }
  bool operator!=(const path &o) const { return s_ != o.s_; }
  bool operator<(const path &o) const { return s_ < o.s_; }

 private:
  std::string s_;
};
inline path operator/(path a, const path &b) { return a /= b; }
inline std::ostream &operator<<(std::ostream &os, const path &p) { return os << p.string(); }
inline bool exists(const path &) { return false; }
inline bool is_regular_file(const path &) { return false; }
inline bool is_directory(const path &) { return false; }

}  // namespace filesystem
}  // namespace boost
