/*
 * Stands in for spdlog when oracle/Makefile compiles reference sources that
 * ask for the "HRRT" logger (spdlog::get): a logger whose methods log
 * nothing.  The LOG_* macros come from oracle/ref_shim.h.  Test
 * infrastructure only.
 */
#pragma once
#include <memory>
#include <string>

namespace spdlog {
class logger {
 public:
  template <class... A> void trace(A &&...) {}
  template <class... A> void debug(A &&...) {}
  template <class... A> void info(A &&...) {}
  template <class... A> void warn(A &&...) {}
  template <class... A> void error(A &&...) {}
  template <class... A> void critical(A &&...) {}
};
inline std::shared_ptr<logger> get(const std::string &) {
  static std::shared_ptr<logger> l = std::make_shared<logger>();
  return l;
}
}  // namespace spdlog
