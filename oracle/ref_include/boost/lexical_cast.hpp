/*
 * Stands in for boost::lexical_cast when oracle/Makefile compiles the
 * reference's listmode histogrammer (named only by the head-curve file
 * parser, which the checkers never call).  Test infrastructure only.
 */
#pragma once
#include <sstream>
#include <string>

namespace boost {
template <class T, class S>
T lexical_cast(const S &s) {
  std::istringstream in(s);
  T v{};
  in >> v;
  return v;
}
}  // namespace boost
