// Host-side tracing: an NVTX range per phase (visible to Nsight tools when
// one is attached; a no-op otherwise) and, when the environment variable
// MSF_TRACE names a file, one JSON line per phase appended to it:
//   {"event": "...", "t": <seconds since the first record>, "seconds": <duration>,
//    "thread": <id>, "detail": "..."}
#pragma once
#include <string>

namespace msf {

class TraceScope {
 public:
  explicit TraceScope(const char* event, std::string detail = std::string());
  ~TraceScope();
  TraceScope(const TraceScope&) = delete;
  TraceScope& operator=(const TraceScope&) = delete;

 private:
  const char* event_;
  std::string detail_;
  double t0_;
};

// Whether MSF_TRACE is set (checked once).
bool trace_enabled();

}  // namespace msf
