/*
 * Minimal stand-in for loguru's `LOG_S(level) << ...` stream macro, which
 * the reference uses for all diagnostics (include/msg.hpp:17).  TEST
 * INFRASTRUCTURE ONLY (see oracle/Makefile.ref).
 *
 * FATAL in the reference aborts the process.  Here it raises a flag that the
 * driver turns into an error status after the stage (results computed after
 * a FATAL are undefined, as in the reference); ERROR and WARNING are counted
 * and the computation continues.  No C++ exception crosses the library.
 */
#ifndef PCG_REF_SHIM_LOGURU_HPP
#define PCG_REF_SHIM_LOGURU_HPP

#include <sstream>
#include <string>

namespace pcg_ref_log {

enum Level { LVL_INFO = 0, LVL_MAX, LVL_WARNING, LVL_ERROR, LVL_FATAL };

// Counters, the fatal flag and the last message, defined in oracle/ref_driver.cpp.
void record(int level, const std::string& msg);

class Line {
 public:
  explicit Line(int level) : level_(level) {}
  template <class T>
  Line& operator<<(const T& v) {
    os_ << v;
    return *this;
  }
  ~Line() { record(level_, os_.str()); }

 private:
  int level_;
  std::ostringstream os_;
};

}  // namespace pcg_ref_log

#define LOG_S(level) pcg_ref_log::Line(pcg_ref_log::LVL_##level)

#endif
