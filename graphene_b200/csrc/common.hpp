// Shared host-side definitions of the graphene_b200 library.
#pragma once

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "../../include/graphene_gpu.h"

namespace gr {

using i32 = int32_t;
using i64 = int64_t;
using u64 = uint64_t;

// Error carried to the C ABI: code is one of the GR_E* values.
struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& msg) : std::runtime_error(msg), code(c) {}
};

[[noreturn]] inline void fail(int code, const std::string& msg) { throw Error(code, msg); }

enum class DType : int { F32 = GR_FLOAT32, F64 = GR_FLOAT64, DW = GR_TWOFLOAT32 };

inline size_t dtypeSize(DType t) {
  switch (t) {
    case DType::F32: return 4;
    case DType::F64: return 8;
    case DType::DW: return 8;
  }
  return 0;
}

inline const char* dtypeName(DType t) {
  switch (t) {
    case DType::F32: return "float32";
    case DType::F64: return "float64";
    case DType::DW: return "twofloat32";
  }
  return "?";
}

template <class T> DType dtypeOf();
template <> inline DType dtypeOf<float>() { return DType::F32; }
template <> inline DType dtypeOf<double>() { return DType::F64; }

inline DType toDType(int t) {
  if (t < 0 || t > 2) fail(GR_EINVAL, "invalid gr_dtype " + std::to_string(t));
  return static_cast<DType>(t);
}

// Host tracing (the reference's GRAPHENE_TRACEPOINT, util/Tracepoint.hpp):
// with GR_TRACE=1 in the environment, every traced scope prints its name and
// wall time to stderr when it ends. Off, a scope costs one cached flag read.
bool traceEnabled();
class TraceScope {
 public:
  explicit TraceScope(const char* name);
  ~TraceScope();
  TraceScope(const TraceScope&) = delete;
  TraceScope& operator=(const TraceScope&) = delete;

 private:
  const char* name_;
  int64_t t0_ = -1;  // steady-clock ns at entry, -1 when tracing is off
};
#define GR_TRACE_CAT2(a, b) a##b
#define GR_TRACE_CAT(a, b) GR_TRACE_CAT2(a, b)
#define GR_TRACE_SCOPE(name) ::gr::TraceScope GR_TRACE_CAT(grTraceScope_, __LINE__)(name)

// Number of host worker threads used by the host pipeline.
inline int hostThreads() {
  unsigned h = std::thread::hardware_concurrency();
  return h == 0 ? 1 : static_cast<int>(std::min(h, 64u));
}

// Runs f(i) for i in [0, n) on up to hostThreads() threads. Tasks are
// handed out dynamically; f must be safe to run concurrently for distinct i.
template <class F>
void parallelFor(i64 n, F&& f) {
  if (n <= 0) return;
  int nt = static_cast<int>(std::min<i64>(hostThreads(), n));
  if (nt <= 1) {
    for (i64 i = 0; i < n; ++i) f(i);
    return;
  }
  std::atomic<i64> next{0};
  std::vector<std::thread> pool;
  std::exception_ptr err = nullptr;
  std::atomic<bool> failed{false};
  pool.reserve(nt);
  for (int t = 0; t < nt; ++t) {
    pool.emplace_back([&]() {
      try {
        for (;;) {
          i64 i = next.fetch_add(1);
          if (i >= n || failed.load()) break;
          f(i);
        }
      } catch (...) {
        if (!failed.exchange(true)) err = std::current_exception();
      }
    });
  }
  for (auto& th : pool) th.join();
  if (err) std::rethrow_exception(err);
}

// Runs f(begin, end) over [0, n) split into contiguous chunks.
template <class F>
void parallelChunks(i64 n, F&& f, i64 minChunk = 1 << 14) {
  if (n <= 0) return;
  i64 nt = std::max<i64>(1, std::min<i64>(hostThreads(), (n + minChunk - 1) / minChunk));
  i64 chunk = (n + nt - 1) / nt;
  parallelFor(nt, [&](i64 t) {
    i64 b = t * chunk, e = std::min(n, b + chunk);
    if (b < e) f(b, e);
  });
}

}  // namespace gr
