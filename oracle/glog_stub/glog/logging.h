/*
 * No-op stand-in for glog, used only to compile the reference's CPU engines
 * into oracle/_ref/ (glog is not installed in this image).  Every LOG/CHECK
 * statement becomes a sink that discards its stream arguments.  Test
 * infrastructure only.
 */
#ifndef ORACLE_GLOG_STUB_LOGGING_H
#define ORACLE_GLOG_STUB_LOGGING_H

#include <ostream>
#include <string>

namespace oracle_glog_stub {
struct Sink {
  template <class T>
  Sink &operator<<(const T &) { return *this; }
  Sink &operator<<(std::ostream &(*)(std::ostream &)) { return *this; }
};
}  // namespace oracle_glog_stub

#define LOG(severity) ::oracle_glog_stub::Sink()
#define CHECK(cond) (void)(cond), ::oracle_glog_stub::Sink()
#define CHECK_EQ(a, b) (void)(a), (void)(b), ::oracle_glog_stub::Sink()

namespace google {
inline void InitGoogleLogging(const char *) {}
inline void InstallFailureSignalHandler() {}
inline void ShutdownGoogleLogging() {}
}  // namespace google

inline std::string FLAGS_log_dir;

#endif
