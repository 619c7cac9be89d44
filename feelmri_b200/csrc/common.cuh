// Shared infrastructure of libfeelmri_b200: context, status handling, launch
// accounting and workspace carving.  Nothing in here computes physics.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <atomic>
#include <string>
#include <vector>

#include "../../include/feelmri_b200.h"

struct fm_timed_launch {
  std::string name;
  cudaEvent_t start, stop;
};

struct fm_ctx {
  int device;
  cudaStream_t stream;
  int num_sms;
  bool timing = false;
  std::vector<fm_timed_launch> timed;
  std::vector<cudaEvent_t> event_pool;
  // helper streams for independent per-problem work forked from `stream` and
  // joined back into it (created on first use), with the fork event and one
  // join event per helper
  std::vector<cudaStream_t> side;
  std::vector<cudaEvent_t> side_ev;
};

namespace fm {

// Thread-local last error (read through fm_last_error).
void set_error(int code, const char *fmt, ...);
int last_code();

extern std::atomic<int64_t> g_launches;
inline void count_launch(int n = 1) { g_launches.fetch_add(n, std::memory_order_relaxed); }

// Returns FM_ERR_CUDA with a message when the last launch failed.
int check_launch(const char *what);

// Makes sure ctx has at least k helper streams (and their events).
int ctx_side_streams(fm_ctx *ctx, int k);
// Work queued on ctx->stream so far comes before anything queued on the
// first k helper streams after this call.
int ctx_fork(fm_ctx *ctx, int k);
// Everything queued on the first k helper streams comes before anything
// queued on ctx->stream after this call.
int ctx_join(fm_ctx *ctx, int k);

#define FM_TRY(expr)                 \
  do {                               \
    int _st = (expr);                \
    if (_st != FM_OK) return _st;    \
  } while (0)

#define FM_CUDA(expr)                                                        \
  do {                                                                       \
    cudaError_t _e = (expr);                                                 \
    if (_e != cudaSuccess) {                                                 \
      ::fm::set_error(FM_ERR_CUDA, "%s failed: %s (%s:%d)", #expr,           \
                      cudaGetErrorString(_e), __FILE__, __LINE__);           \
      return FM_ERR_CUDA;                                                    \
    }                                                                        \
  } while (0)

#define FM_REQUIRE(cond, code, ...)          \
  do {                                       \
    if (!(cond)) {                           \
      ::fm::set_error((code), __VA_ARGS__);  \
      return (code);                         \
    }                                        \
  } while (0)

// Makes the context's device current for the duration of an entry point.
struct DeviceGuard {
  int prev = -1;
  bool ok = true;
  explicit DeviceGuard(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (prev != dev) ok = (cudaSetDevice(dev) == cudaSuccess);
  }
  ~DeviceGuard() {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
};

// Bump allocator over a caller-provided workspace.  When base is null it only
// measures (the *_workspace_size queries run the same carving code).
struct Carve {
  char *base;
  size_t cap;
  size_t used = 0;
  bool overflow = false;
  Carve(void *b, size_t c) : base(static_cast<char *>(b)), cap(c) {}
  template <class T>
  T *take(size_t count, size_t align = 256) {
    size_t off = (used + align - 1) / align * align;
    size_t bytes = count * sizeof(T);
    used = off + bytes;
    if (base == nullptr) return nullptr;
    if (used > cap) {
      overflow = true;
      return nullptr;
    }
    return reinterpret_cast<T *>(base + off);
  }
};

inline int carve_ok(const Carve &c, const char *what) {
  if (c.overflow) {
    set_error(FM_ERR_NOMEM, "%s: workspace too small (%zu bytes given, %zu needed)", what, c.cap, c.used);
    return FM_ERR_NOMEM;
  }
  return FM_OK;
}

inline int ctx_ok(const fm_ctx *ctx) {
  if (ctx == nullptr) {
    set_error(FM_ERR_ARG, "null fm_ctx");
    return FM_ERR_ARG;
  }
  return FM_OK;
}

__host__ __device__ inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }

// Records a start event for a named launch when timing is enabled; returns
// the slot to pass to timer_stop (or -1).
int timer_start(fm_ctx *ctx, const char *name);
void timer_stop(fm_ctx *ctx, int slot);

struct ScopedTimer {
  fm_ctx *ctx;
  int slot;
  ScopedTimer(fm_ctx *c, const char *name) : ctx(c), slot(timer_start(c, name)) {}
  ~ScopedTimer() { timer_stop(ctx, slot); }
};

}  // namespace fm
