// Stand-in for easylogging++ when the reference's code generator is compiled for the oracle cross-check
// (TEST INFRASTRUCTURE ONLY).  LOG/VLOG statements are swallowed; LOG(FATAL) throws so that a failing
// generation stops the driver with the message.  The standard headers the real library brings along (and
// the generator's sources rely on) are included here.
#pragma once
#include <fstream>
#include <functional>
#include <iostream>
#include <list>
#include <map>
#include <set>
#include <sstream>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

namespace refgen_log {
template<class T, class = void>
struct streamable : std::false_type {};
template<class T>
struct streamable<T, std::void_t<decltype(std::declval<std::ostream&>() << std::declval<const T&>())>>
    : std::true_type {};

struct Sink {
  bool fatal;
  std::ostringstream s;
  explicit Sink(bool f) : fatal(f) {}
  ~Sink() noexcept(false)
  {
    if (fatal)
      throw std::runtime_error(s.str());
  }
  template<class T>
  Sink& operator<<(const T& v)
  {
    if constexpr (streamable<T>::value) {
      if (fatal)
        s << v;
    }
    return *this;
  }
  Sink& operator<<(std::ostream& (*)(std::ostream&)) { return *this; }
};
} // namespace refgen_log

#define REFGEN_LOG_INFO refgen_log::Sink(false)
#define REFGEN_LOG_DEBUG refgen_log::Sink(false)
#define REFGEN_LOG_WARNING refgen_log::Sink(false)
#define REFGEN_LOG_ERROR refgen_log::Sink(false)
#define REFGEN_LOG_TRACE refgen_log::Sink(false)
#define REFGEN_LOG_FATAL refgen_log::Sink(true)
#define LOG(level) REFGEN_LOG_##level
#define VLOG(n) refgen_log::Sink(false)
#define VLOG_IS_ON(n) false
