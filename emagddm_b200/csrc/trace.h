// trace.h -- opt-in host-side phase tracing (set EMG_TRACE=1): every traced
// scope prints its wall time to stderr as "emg-trace <name> <ms>".
#pragma once

#include <chrono>
#include <cstdio>
#include <cstdlib>

namespace emg {

inline bool trace_enabled() {
  static const bool on = [] {
    const char* v = std::getenv("EMG_TRACE");
    return v && v[0] && v[0] != '0';
  }();
  return on;
}

// With tracing on: the reserved and used bytes of the current device's
// default stream-ordered memory pool, as "emg-trace-pool <where> <reserved> <used>".
void trace_pool(const char* where);
// With tracing on: synchronizes the stream (a cudaStream_t) and prints the
// wall time since the previous mark of this thread, "emg-trace-mark <label> <ms>".
void trace_mark(void* stream, const char* label);

class TraceScope {
 public:
  explicit TraceScope(const char* name) : name_(name) {
    if (trace_enabled()) t0_ = std::chrono::steady_clock::now();
  }
  ~TraceScope() {
    if (!trace_enabled()) return;
    const double ms =
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0_).count();
    std::fprintf(stderr, "emg-trace %s %.3f\n", name_, ms);
  }

 private:
  const char* name_;
  std::chrono::steady_clock::time_point t0_{};
};

}  // namespace emg
