// Host-side tracing (trace.hpp).
#include "trace.hpp"

#include <nvtx3/nvToolsExt.h>

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <functional>
#include <mutex>
#include <thread>

namespace msf {

namespace {

struct Sink {
  std::FILE* f = nullptr;
  std::mutex m;
  std::chrono::steady_clock::time_point origin = std::chrono::steady_clock::now();
  Sink() {
    if (const char* path = std::getenv("MSF_TRACE"))
      if (*path) f = std::fopen(path, "a");
  }
  ~Sink() {
    if (f) std::fclose(f);
  }
};

Sink& sink() {
  static Sink s;
  return s;
}

double now() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - sink().origin).count();
}

std::string escaped(const std::string& s) {
  std::string o;
  for (char c : s) {
    if (c == '"' || c == '\\') o.push_back('\\');
    if ((unsigned char)c >= 0x20) o.push_back(c);
  }
  return o;
}

}  // namespace

bool trace_enabled() { return sink().f != nullptr; }

TraceScope::TraceScope(const char* event, std::string detail)
    : event_(event), detail_(std::move(detail)), t0_(now()) {
  nvtxRangePushA(event);
}

TraceScope::~TraceScope() {
  nvtxRangePop();
  Sink& s = sink();
  if (!s.f) return;
  const double t1 = now();
  const size_t tid = std::hash<std::thread::id>()(std::this_thread::get_id()) % 1000000;
  std::lock_guard<std::mutex> lock(s.m);
  std::fprintf(s.f,
               "{\"event\": \"%s\", \"t\": %.6f, \"seconds\": %.6f, \"thread\": %zu, "
               "\"detail\": \"%s\"}\n",
               event_, t0_, t1 - t0_, tid, escaped(detail_).c_str());
  std::fflush(s.f);
}

}  // namespace msf
