// Minimal stand-in for the {fmt} library, enough for the reference's logging
// calls on the path tracing route (fmt::print / fmt::format with "{}" and
// "{:.Nf}" placeholders). Test infrastructure for the reference oracle build.
#pragma once
#include <cstdio>
#include <sstream>
#include <string>
#include <iomanip>
#include <iostream>

#define FMT_BEGIN_NAMESPACE namespace fmt {
#define FMT_END_NAMESPACE }

namespace fmt {
struct ostream_formatter {};
template <typename T> struct formatter {};

namespace detail {
inline void emit(std::ostringstream& os, const std::string& f, size_t& pos) {
  os << f.substr(pos);
  pos = f.size();
}
template <typename T, typename... Rest>
void emit(std::ostringstream& os, const std::string& f, size_t& pos, const T& v, const Rest&... rest) {
  size_t open = f.find('{', pos);
  if (open == std::string::npos) { os << f.substr(pos); pos = f.size(); return; }
  size_t close = f.find('}', open);
  os << f.substr(pos, open - pos);
  std::string spec = f.substr(open + 1, close - open - 1);
  std::ostringstream one;
  if (spec.size() > 2 && spec[0] == ':' && spec[1] == '.') {
    int prec = std::atoi(spec.c_str() + 2);
    one << std::fixed << std::setprecision(prec);
  }
  one << v;
  os << one.str();
  pos = close + 1;
  emit(os, f, pos, rest...);
}
}  // namespace detail

template <typename... Args>
std::string format(const std::string& f, const Args&... args) {
  std::ostringstream os;
  size_t pos = 0;
  detail::emit(os, f, pos, args...);
  return os.str();
}
template <typename... Args>
void print(const std::string& f, const Args&... args) {
  std::string s = format(f, args...);
  std::fwrite(s.data(), 1, s.size(), stdout);
}
}  // namespace fmt
